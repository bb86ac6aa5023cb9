// libgrimgpu: C-ABI exports and host orchestration of the B200 RCS solve path.
// One translation unit (constant-memory tables are shared by every kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "fill2d.cuh"
#include "hankel.cuh"
#include "linalg.cuh"
#include "lu.cuh"
#include "bor.cuh"
#include "tc_gemm.cuh"
#include "ozaki.cuh"
#include "dmma.cuh"
#include "grouped.cuh"
#include "farblock.cuh"
#include "galerkin.cuh"
#include "pivot.cuh"
#include "tslu.cuh"
#include "gepp_loop.cuh"
#include "condest.cuh"
#include "modecond.cuh"

// ============================================================== errors
static thread_local std::string g_last_error;

void grim_set_error(const std::string &msg) { g_last_error = msg; }
int grim_fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
int grim_cuda_check(cudaError_t e, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? GRIM_ERR_NOMEM : GRIM_ERR_CUDA;
}

// ============================================================== tables
// Gauss-Legendre nodes by Newton iteration on P_q (three-term recurrence), weights
// 2 / ((1 - x^2) P_q'(x)^2).
static void gauss_legendre(int q, double *x, double *w) {
    for (int i = 0; i < q; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (q + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int l = 2; l <= q; ++l) {
                const double p2 = ((2.0 * l - 1.0) * z * p1 - (l - 1.0) * p0) / l;
                p0 = p1;
                p1 = p2;
            }
            if (q == 1) { p1 = z; p0 = 1.0; }
            dp = q * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) {
                // one more polish step
                p0 = 1.0; p1 = z;
                for (int l = 2; l <= q; ++l) {
                    const double p2 = ((2.0 * l - 1.0) * z * p1 - (l - 1.0) * p0) / l;
                    p0 = p1;
                    p1 = p2;
                }
                if (q == 1) { p1 = z; p0 = 1.0; }
                dp = q * (z * p1 - p0) / (z * z - 1.0);
                break;
            }
        }
        // nodes ascending
        x[q - 1 - i] = z;
        w[q - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
    if (q == 1) { x[0] = 0.0; w[0] = 2.0; }
}

static std::mutex g_table_mutex;
static std::vector<int> g_tables_ready;  // per device

static int upload_tables(int device) {
    std::lock_guard<std::mutex> lk(g_table_mutex);
    if ((int)g_tables_ready.size() <= device) g_tables_ready.resize(device + 1, 0);
    if (g_tables_ready[device]) return GRIM_OK;
    std::vector<double> gx(GRIM_MAX_GAUSS * (GRIM_MAX_GAUSS + 1) / 2), gw(gx.size());
    for (int q = 1; q <= GRIM_MAX_GAUSS; ++q) gauss_legendre(q, &gx[q * (q - 1) / 2], &gw[q * (q - 1) / 2]);
    GRIM_CHECK_CUDA(cudaMemcpyToSymbol(c_gl_x, gx.data(), gx.size() * sizeof(double)));
    GRIM_CHECK_CUDA(cudaMemcpyToSymbol(c_gl_w, gw.data(), gw.size() * sizeof(double)));
    float a0[GRIM_ASYM_TERMS], a1[GRIM_ASYM_TERMS];
    double d0 = 1.0, d1 = 1.0;
    for (int kk = 0; kk < GRIM_ASYM_TERMS; ++kk) {
        if (kk > 0) {
            const double odd = (2.0 * kk - 1.0) * (2.0 * kk - 1.0);
            d0 *= (0.0 - odd) / (8.0 * kk);
            d1 *= (4.0 - odd) / (8.0 * kk);
        }
        a0[kk] = (float)d0;
        a1[kk] = (float)d1;
    }
    GRIM_CHECK_CUDA(cudaMemcpyToSymbol(c_asym_a0, a0, sizeof(a0)));
    GRIM_CHECK_CUDA(cudaMemcpyToSymbol(c_asym_a1, a1, sizeof(a1)));
    double g0[GAL_ASYM64_TERMS], g1[GAL_ASYM64_TERMS];
    g0[0] = g1[0] = 1.0;
    for (int kk = 1; kk < GAL_ASYM64_TERMS; ++kk) {
        const double odd = (2.0 * kk - 1.0) * (2.0 * kk - 1.0);
        g0[kk] = g0[kk - 1] * (0.0 - odd) / (8.0 * kk);
        g1[kk] = g1[kk - 1] * (4.0 - odd) / (8.0 * kk);
    }
    GRIM_CHECK_CUDA(cudaMemcpyToSymbol(c_gal_a0, g0, sizeof(g0)));
    GRIM_CHECK_CUDA(cudaMemcpyToSymbol(c_gal_a1, g1, sizeof(g1)));
    g_tables_ready[device] = 1;
    return GRIM_OK;
}

int grim_upload_gauss(void) {
    int dev = 0;
    cudaGetDevice(&dev);
    return upload_tables(dev);
}

// Status-returning form of GRIM_CHECK_LAUNCH_W, for code that must clean up on failure.
int grim_launch_status(grim_context *h, const char *what, double flops, double bytes) {
    h->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return grim_cuda_check(e, what);
    if (h->profiling) grim_prof_mark(h, what, flops, bytes);
    return GRIM_OK;
}
int grim_cuda_status(cudaError_t e, const char *what) { return e == cudaSuccess ? GRIM_OK : grim_cuda_check(e, what); }

// ============================================================== workspace
int grim_workspace(grim_context *h, const char *name, size_t bytes, void **out) {
    auto it = h->ws.find(name);
    if (it != h->ws.end() && it->second.second >= bytes) {
        *out = it->second.first;
        return GRIM_OK;
    }
    if (it != h->ws.end()) {
        GRIM_CHECK_CUDA(cudaFreeAsync(it->second.first, h->stream));
        h->ws.erase(it);
    }
    void *p = nullptr;
    const size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMallocAsync(&p, want, h->stream);
    if (e != cudaSuccess) return grim_cuda_check(e, "workspace allocation");
    h->ws[name] = {p, want};
    *out = p;
    return GRIM_OK;
}

// ============================================================== context API
extern "C" int grim_version(void) { return 1; }
extern "C" const char *grim_last_error(void) { return g_last_error.c_str(); }

extern "C" int grim_create(int device, grim_handle_t *out) {
    if (!out) return grim_fail(GRIM_ERR_ARGUMENT, "grim_create: null output pointer");
    int count = 0;
    GRIM_CHECK_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return grim_fail(GRIM_ERR_ARGUMENT, "grim_create: no such CUDA device");
    DeviceGuard g(device);
    auto *h = new grim_context();
    h->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return grim_cuda_check(e, "cudaStreamCreate");
    }
    h->stream = h->own_stream;
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
    int s = upload_tables(device);
    if (s != GRIM_OK) {
        cudaStreamDestroy(h->own_stream);
        delete h;
        return s;
    }
    *out = h;
    return GRIM_OK;
}

extern "C" int grim_release_workspace(grim_handle_t h) {
    if (!h) return grim_fail(GRIM_ERR_ARGUMENT, "null handle");
    DeviceGuard g(h->device);
    for (auto &kv : h->ws) cudaFreeAsync(kv.second.first, h->stream);
    h->ws.clear();
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (h->grp_exec) {  // the captured grouped factorization read the freed buffers
        cudaGraphExecDestroy(h->grp_exec);
        h->grp_exec = nullptr;
        h->grp_key.clear();
    }
    return GRIM_OK;
}

extern "C" int grim_destroy(grim_handle_t h) {
    if (!h) return GRIM_OK;
    DeviceGuard g(h->device);
    grim_release_workspace(h);
    if (h->tc_err) {
        cudaStreamSynchronize(h->stream);
        cudaFree(h->tc_err);
    }
    if (h->chain) cudaStreamSynchronize(h->chain);
    if (h->bulk) cudaStreamSynchronize(h->bulk);
    for (cudaEvent_t e : h->events) cudaEventDestroy(e);
    if (h->chain) cudaStreamDestroy(h->chain);
    if (h->bulk) cudaStreamDestroy(h->bulk);
    if (h->grp_exec) cudaGraphExecDestroy(h->grp_exec);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return GRIM_OK;
}

extern "C" int grim_set_stream(grim_handle_t h, void *stream) {
    if (!h) return grim_fail(GRIM_ERR_ARGUMENT, "null handle");
    // NULL is CUDA's default (legacy) stream, which is where PyTorch runs by default.
    h->stream = (cudaStream_t)stream;
    return GRIM_OK;
}
extern "C" void *grim_get_stream(grim_handle_t h) { return h ? (void *)h->stream : nullptr; }
static int tc_err_check(grim_context *h, const char *what);
extern "C" int grim_synchronize(grim_handle_t h) {
    if (!h) return grim_fail(GRIM_ERR_ARGUMENT, "null handle");
    DeviceGuard g(h->device);
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return tc_err_check(h, "a tensor-core kernel since the last check");
}
extern "C" int64_t grim_launch_count(grim_handle_t h) { return h ? h->launches : 0; }
extern "C" int grim_device_name(grim_handle_t h, char *buf, int len) {
    if (!h || !buf || len <= 0) return grim_fail(GRIM_ERR_ARGUMENT, "grim_device_name: bad arguments");
    cudaDeviceProp p;
    GRIM_CHECK_CUDA(cudaGetDeviceProperties(&p, h->device));
    std::snprintf(buf, (size_t)len, "%s", p.name);
    return GRIM_OK;
}
extern "C" int grim_mem_info(grim_handle_t h, size_t *free_bytes, size_t *total_bytes) {
    if (!h || !free_bytes || !total_bytes) return grim_fail(GRIM_ERR_ARGUMENT, "grim_mem_info: bad arguments");
    DeviceGuard g(h->device);
    GRIM_CHECK_CUDA(cudaMemGetInfo(free_bytes, total_bytes));
    return GRIM_OK;
}
extern "C" int grim_set_tuning(grim_handle_t h, int key, int value) {
    if (!h) return grim_fail(GRIM_ERR_ARGUMENT, "null handle");
    if (key == GRIM_TUNE_SOLVE_BN && (value == 0 || value == 64 || value == 128)) {
        h->tune_solve_bn = value;
        return GRIM_OK;
    }
    if (key == GRIM_TUNE_GS_BLOCK && (value == 0 || value == 64 || value == 128 || value == 256 || value == 512)) {
        h->tune_gs_block = value;
        return GRIM_OK;
    }
    if (key == GRIM_TUNE_PIVOT && value >= GRIM_PIVOT_CERTIFIED && value <= GRIM_PIVOT_TOURNAMENT) {
        h->pivot_mode = value;
        return GRIM_OK;
    }
    return grim_fail(GRIM_ERR_ARGUMENT, "grim_set_tuning: unknown key or value out of range");
}

extern "C" int grim_last_solve_info(grim_handle_t h, grim_solve_info *out) {
    if (!h || !out) return grim_fail(GRIM_ERR_ARGUMENT, "grim_last_solve_info: bad arguments");
    *out = h->last;
    return GRIM_OK;
}

// ============================================================== 2-D fill / rhs / far field
extern "C" int grim_fill2d(grim_handle_t h, int pol, int n, const double *geom, const double *diag_extra, double k,
                           void *Z, int64_t ldz, int out_complex64) {
    if (!h || n <= 0 || !geom || !Z || ldz < n || !(k > 0) || (pol != GRIM_POL_TM && pol != GRIM_POL_TE))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_fill2d: bad arguments");
    DeviceGuard g(h->device);
    dim3 grid(ceil_div(n, FILL_ROWS), ceil_div(n, FILL_COLS));
    dim3 block(FILL_ROWS * FILL_WARPS);
    if (out_complex64) {
        if (pol == GRIM_POL_TM)
            k_fill2d<GRIM_POL_TM, float2><<<grid, block, 0, h->stream>>>(n, geom, diag_extra, k, (float2 *)Z, ldz);
        else
            k_fill2d<GRIM_POL_TE, float2><<<grid, block, 0, h->stream>>>(n, geom, diag_extra, k, (float2 *)Z, ldz);
    } else {
        if (pol == GRIM_POL_TM)
            k_fill2d<GRIM_POL_TM, double2><<<grid, block, 0, h->stream>>>(n, geom, diag_extra, k, (double2 *)Z, ldz);
        else
            k_fill2d<GRIM_POL_TE, double2><<<grid, block, 0, h->stream>>>(n, geom, diag_extra, k, (double2 *)Z, ldz);
    }
    GRIM_CHECK_LAUNCH(h, "k_fill2d");
    return GRIM_OK;
}

extern "C" int grim_rhs2d(grim_handle_t h, int pol, int n, const double *geom, int nang, const double *angles_deg,
                          double k, void *B, int64_t ldb, int out_complex64) {
    if (!h || n <= 0 || nang <= 0 || !geom || !angles_deg || !B || ldb < n || nang > 65535 ||
        (pol != GRIM_POL_TM && pol != GRIM_POL_TE))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_rhs2d: bad arguments");
    DeviceGuard g(h->device);
    dim3 grid(ceil_div(n, 256), nang);
    if (out_complex64) {
        if (pol == GRIM_POL_TM) k_rhs2d<GRIM_POL_TM, float2><<<grid, 256, 0, h->stream>>>(n, geom, nang, angles_deg, k, (float2 *)B, ldb);
        else k_rhs2d<GRIM_POL_TE, float2><<<grid, 256, 0, h->stream>>>(n, geom, nang, angles_deg, k, (float2 *)B, ldb);
    } else {
        if (pol == GRIM_POL_TM) k_rhs2d<GRIM_POL_TM, double2><<<grid, 256, 0, h->stream>>>(n, geom, nang, angles_deg, k, (double2 *)B, ldb);
        else k_rhs2d<GRIM_POL_TE, double2><<<grid, 256, 0, h->stream>>>(n, geom, nang, angles_deg, k, (double2 *)B, ldb);
    }
    GRIM_CHECK_LAUNCH(h, "k_rhs2d");
    return GRIM_OK;
}

extern "C" int grim_farfield2d(grim_handle_t h, int n, const double *geom, int nang, const double *angles_deg, double k,
                               const void *X, int64_t ldx, int x_complex64, void *amp) {
    if (!h || n <= 0 || nang <= 0 || !geom || !angles_deg || !X || !amp || ldx < n)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_farfield2d: bad arguments");
    DeviceGuard g(h->device);
    if (x_complex64)
        k_farfield2d<float2><<<nang, 256, 0, h->stream>>>(n, geom, nang, angles_deg, k, (const float2 *)X, ldx, (double2 *)amp);
    else
        k_farfield2d<double2><<<nang, 256, 0, h->stream>>>(n, geom, nang, angles_deg, k, (const double2 *)X, ldx, (double2 *)amp);
    GRIM_CHECK_LAUNCH(h, "k_farfield2d");
    return GRIM_OK;
}

// ============================================================== linear-Galerkin fill
static bool gal_elem_ok(int ne, const double *elem, const int *nodes) { return ne > 0 && elem && nodes; }

extern "C" int grim_gal_near_count(grim_handle_t h, int ne, const double *elem, const int *nodes, int *row_off,
                                   int *nnz_host) {
    if (!h || !gal_elem_ok(ne, elem, nodes) || !row_off || !nnz_host)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_gal_near_count: bad arguments");
    DeviceGuard g(h->device);
    void *pc = nullptr;
    GRIM_TRY(grim_workspace(h, "gal_count", (size_t)ne * sizeof(int), &pc));
    const int wpb = 8;
    k_gal_near_count<<<ceil_div(ne, wpb), 32 * wpb, 0, h->stream>>>(ne, elem, (const int2 *)nodes, (int *)pc);
    GRIM_CHECK_LAUNCH(h, "k_gal_near_count");
    k_gal_scan<<<1, 1024, 0, h->stream>>>(ne, (const int *)pc, row_off);
    GRIM_CHECK_LAUNCH(h, "k_gal_scan");
    GRIM_CHECK_CUDA(cudaMemcpyAsync(nnz_host, row_off + ne, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return GRIM_OK;
}

extern "C" int grim_gal_near_list(grim_handle_t h, int ne, const double *elem, const int *nodes, const int *row_off,
                                  int *col, int *route) {
    if (!h || !gal_elem_ok(ne, elem, nodes) || !row_off || !col || !route)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_gal_near_list: bad arguments");
    DeviceGuard g(h->device);
    const int wpb = 8;
    k_gal_near_list<<<ceil_div(ne, wpb), 32 * wpb, 0, h->stream>>>(ne, elem, (const int2 *)nodes, row_off, col, route);
    GRIM_CHECK_LAUNCH(h, "k_gal_near_list");
    return GRIM_OK;
}

static int gal_err_flag(grim_context *h, int **out) {
    void *p = nullptr;
    const bool fresh = h->ws.find("gal_err") == h->ws.end();
    GRIM_TRY(grim_workspace(h, "gal_err", sizeof(int), &p));
    if (fresh) GRIM_CHECK_CUDA(cudaMemsetAsync(p, 0, sizeof(int), h->stream));
    *out = (int *)p;
    return GRIM_OK;
}

static int lookahead_streams(grim_context *h, int nevents);

template <typename C>
static int gal_fill_impl(grim_context *h, int pol, int ne, int n, const double *elem, const int2 *nodes,
                         const int *start_of, const int *end_of, const int *row_off, const int *col, const int *route,
                         int nnz, const int *adapt_idx, int nadapt, double k, int far_min_order, C *Z, int64_t ldz) {
    void *pnb = nullptr, *pe = nullptr, *pst = nullptr;
    int *err = nullptr;
    GRIM_TRY(gal_err_flag(h, &err));
    GRIM_TRY(grim_workspace(h, "gal_nb", (size_t)nnz * 8 * sizeof(double2), &pnb));
    GRIM_TRY(grim_workspace(h, "gal_e", (size_t)ne * ne * 4 * sizeof(C), &pe));
    if (nadapt > 0)
        GRIM_TRY(grim_workspace(h, "gal_adapt_stack", (size_t)nadapt * GAL_ADAPT_GCAP * sizeof(GalBox), &pst));
    double2 *nbk = (double2 *)pnb;
    C *E = (C *)pe;
    // The near pairs (k_gal_near, k_gal_adapt: NBK) and the far pairs (k_gal_far: E) write
    // disjoint buffers, so the near work -- the adaptive close pairs are a few hundred
    // long-running CTAs -- runs on the handle's high-priority stream beside the far tiles
    // (not when profiling per launch); the near routing waits for both.
    const bool split = !h->profiling;
    const cudaStream_t caller = h->stream;
    if (split) {
        GRIM_TRY(lookahead_streams(h, 2));
        GRIM_CHECK_CUDA(cudaEventRecord(h->events[0], caller));
        GRIM_CHECK_CUDA(cudaStreamWaitEvent(h->chain, h->events[0], 0));
        h->stream = h->chain;
    }
    int status = GRIM_OK;
    k_gal_near<<<ceil_div(nnz, GAL_NEAR_WARPS), GAL_NEAR_WARPS * 32, 0, h->stream>>>(ne, nnz, elem, nodes, row_off,
                                                                                     col, route, k, nbk, err);
    status = grim_launch_status(h, "k_gal_near", 0, 0);
    if (status == GRIM_OK && nadapt > 0) {
        static PerDeviceOnce attr;
        if (attr.needed()) {
            cudaError_t e = cudaFuncSetAttribute(k_gal_adapt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)GAL_ADAPT_SMEM);
            if (e != cudaSuccess) status = grim_cuda_check(e, "k_gal_adapt attribute");
            else attr.mark();
        }
        if (status == GRIM_OK) {
            k_gal_adapt<<<nadapt, GAL_ADAPT_WARPS * 32, GAL_ADAPT_SMEM, h->stream>>>(ne, nadapt, adapt_idx, elem,
                                                                                       row_off, col, k, (GalBox *)pst,
                                                                                       nbk, err);
            status = grim_launch_status(h, "k_gal_adapt", 0, 0);
        }
    }
    if (split) {
        // the caller's stream carries on with the far tiles, then waits for the near work
        cudaEventRecord(h->events[1], h->chain);
        h->stream = caller;
    }
    if (status != GRIM_OK) {
        if (split) cudaStreamWaitEvent(caller, h->events[1], 0);
        return status;
    }
    const int tiles = ceil_div(ne, GAL_TILE);
    dim3 fg(tiles, tiles);
    if (pol == GRIM_POL_TM)
        k_gal_far<GRIM_POL_TM, C><<<fg, GAL_FAR_THREADS, 0, h->stream>>>(ne, elem, nodes, k, far_min_order, E);
    else
        k_gal_far<GRIM_POL_TE, C><<<fg, GAL_FAR_THREADS, 0, h->stream>>>(ne, elem, nodes, k, far_min_order, E);
    status = grim_launch_status(h, "k_gal_far", 0, 0);
    if (split) GRIM_CHECK_CUDA(cudaStreamWaitEvent(caller, h->events[1], 0));
    GRIM_TRY(status);
    if (pol == GRIM_POL_TM)
        k_gal_near_route<GRIM_POL_TM, C><<<ceil_div(nnz, 128), 128, 0, h->stream>>>(ne, nnz, elem, row_off, col, nbk, k, E);
    else
        k_gal_near_route<GRIM_POL_TE, C><<<ceil_div(nnz, 128), 128, 0, h->stream>>>(ne, nnz, elem, row_off, col, nbk, k, E);
    GRIM_CHECK_LAUNCH(h, "k_gal_near_route");
    dim3 gg(ceil_div(n, 128), n);
    k_gal_gather<C><<<gg, 128, 0, h->stream>>>(ne, n, start_of, end_of, E, Z, ldz);
    GRIM_CHECK_LAUNCH(h, "k_gal_gather");
    return GRIM_OK;
}

extern "C" int grim_gal_fill(grim_handle_t h, int pol, int ne, int n, const double *elem, const int *nodes,
                             const int *start_of, const int *end_of, const int *row_off, const int *col,
                             const int *route, int nnz, const int *adapt_idx, int nadapt, double k,
                             int far_min_order, void *Z, int64_t ldz, int out_complex64) {
    if (!h || !gal_elem_ok(ne, elem, nodes) || n <= 0 || n > 65535 || !start_of || !end_of || !row_off || !col ||
        !route || nnz < ne || nadapt < 0 || (nadapt > 0 && !adapt_idx) || !Z || ldz < n || !(k > 0) ||
        far_min_order < 0 || far_min_order > GAL_MAX_Q || (pol != GRIM_POL_TM && pol != GRIM_POL_TE))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_gal_fill: bad arguments");
    DeviceGuard g(h->device);
    if (out_complex64)
        return gal_fill_impl<float2>(h, pol, ne, n, elem, (const int2 *)nodes, start_of, end_of, row_off, col, route,
                                     nnz, adapt_idx, nadapt, k, far_min_order, (float2 *)Z, ldz);
    return gal_fill_impl<double2>(h, pol, ne, n, elem, (const int2 *)nodes, start_of, end_of, row_off, col, route,
                                  nnz, adapt_idx, nadapt, k, far_min_order, (double2 *)Z, ldz);
}

extern "C" int grim_gal_status(grim_handle_t h, int *flag_host) {
    if (!h || !flag_host) return grim_fail(GRIM_ERR_ARGUMENT, "grim_gal_status: bad arguments");
    DeviceGuard g(h->device);
    int *err = nullptr;
    GRIM_TRY(gal_err_flag(h, &err));
    GRIM_CHECK_CUDA(cudaMemcpyAsync(flag_host, err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return GRIM_OK;
}

extern "C" int grim_gal_rhs(grim_handle_t h, int pol, int n, const double *elem, const int *start_of,
                            const int *end_of, int nang, const double *angles_deg, double k, void *B, int64_t ldb,
                            int out_complex64) {
    if (!h || n <= 0 || !elem || !start_of || !end_of || nang <= 0 || nang > 65535 || !angles_deg || !B || ldb < n ||
        !(k > 0) || (pol != GRIM_POL_TM && pol != GRIM_POL_TE))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_gal_rhs: bad arguments");
    DeviceGuard g(h->device);
    dim3 grid(ceil_div(n, 128), nang);
#define GAL_RHS(P, C) k_gal_rhs<P, C><<<grid, 128, 0, h->stream>>>(n, elem, start_of, end_of, nang, angles_deg, k, (C *)B, ldb)
    if (out_complex64) {
        if (pol == GRIM_POL_TM) GAL_RHS(GRIM_POL_TM, float2);
        else GAL_RHS(GRIM_POL_TE, float2);
    } else {
        if (pol == GRIM_POL_TM) GAL_RHS(GRIM_POL_TM, double2);
        else GAL_RHS(GRIM_POL_TE, double2);
    }
#undef GAL_RHS
    GRIM_CHECK_LAUNCH(h, "k_gal_rhs");
    return GRIM_OK;
}

extern "C" int grim_gal_farfield(grim_handle_t h, int ne, const double *elem, const int *nodes, int nang,
                                 const double *angles_deg, double k, const void *X, int64_t ldx, int x_complex64,
                                 void *amp) {
    if (!h || !gal_elem_ok(ne, elem, nodes) || nang <= 0 || !angles_deg || !X || !amp || !(k > 0))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_gal_farfield: bad arguments");
    DeviceGuard g(h->device);
    if (x_complex64)
        k_gal_farfield<float2><<<nang, 256, 0, h->stream>>>(ne, elem, (const int2 *)nodes, nang, angles_deg, k,
                                                            (const float2 *)X, ldx, (double2 *)amp);
    else
        k_gal_farfield<double2><<<nang, 256, 0, h->stream>>>(ne, elem, (const int2 *)nodes, nang, angles_deg, k,
                                                             (const double2 *)X, ldx, (double2 *)amp);
    GRIM_CHECK_LAUNCH(h, "k_gal_farfield");
    return GRIM_OK;
}

// ============================================================== GEMM launcher
static int tc_enabled();

template <bool NEG, bool BETA>
static int dmma_gemm(grim_context *h, int M, int N, int K, const double2 *A, int64_t lda, const double2 *B,
                     int64_t ldb, double2 *C, int64_t ldc) {
    static PerDeviceOnce attr;
    if (attr.needed()) {
        GRIM_CHECK_CUDA(
            cudaFuncSetAttribute(k_gemm_dmma<NEG, BETA>, cudaFuncAttributeMaxDynamicSharedMemorySize, DM_SMEM_BYTES));
        attr.mark();
    }
    dim3 grid(ceil_div(M, DM_BM), ceil_div(N, DM_BN));
    k_gemm_dmma<NEG, BETA><<<grid, DM_THREADS, DM_SMEM_BYTES, h->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
    GRIM_CHECK_LAUNCH_W(h, "k_gemm_dmma", 8.0 * M * N * K, 16.0 * ((double)M * K + (double)K * N + 2.0 * M * N));
    return GRIM_OK;
}

// C = (BETA ? C : 0) + (NEG ? -1 : 1) A B.  Complex128 throughout: FP64 tensor cores
// (k_gemm_dmma) unless disabled; other type mixes: the SIMT register-tiled kernel.
template <typename ACC, typename TA, typename TB, typename TC, bool NEG, bool BETA>
static int gemm(grim_context *h, int M, int N, int K, const TA *A, int64_t lda, const TB *B, int64_t ldb, TC *C,
                int64_t ldc) {
    if (M <= 0 || N <= 0) return GRIM_OK;
    if constexpr (sizeof(ACC) == 16 && sizeof(TA) == 16 && sizeof(TB) == 16 && sizeof(TC) == 16) {
        if (tc_enabled() && K > 0)
            return dmma_gemm<NEG, BETA>(h, M, N, K, (const double2 *)A, lda, (const double2 *)B, ldb, (double2 *)C,
                                        ldc);
    }
    dim3 grid(ceil_div(M, RT_BM), ceil_div(N, RT_BN));
    k_gemm_rt<ACC, TA, TB, TC, NEG, BETA><<<grid, RT_THREADS, 0, h->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, 0, 0,
                                                                              0);
    GRIM_CHECK_LAUNCH_W(h, sizeof(ACC) == 16 ? "k_gemm_rt<f64>" : "k_gemm_rt<f32>", 8.0 * M * N * K,
                        (double)sizeof(TA) * M * K + (double)sizeof(TB) * K * N + (BETA ? 2.0 : 1.0) * sizeof(TC) * M * N);
    return GRIM_OK;
}

// ============================================================== tensor-core complex64 update
static int tc_enabled() {
    static int v = -1;
    if (v < 0) {
        const char *e = std::getenv("GRIM_TENSOR_CORES");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v;
}

// Device error flag of the tensor-core kernels: zeroed once per context; a set flag is
// reported (and cleared) by the next tc_err_check.
static int tc_err_flag(grim_context *h, int **out) {
    if (!h->tc_err) {
        void *p = nullptr;
        GRIM_CHECK_CUDA(cudaMalloc(&p, sizeof(int)));
        GRIM_CHECK_CUDA(cudaMemsetAsync(p, 0, sizeof(int), h->stream));
        h->tc_err = (int *)p;
    }
    *out = h->tc_err;
    return GRIM_OK;
}

// Host read of the flag (synchronises the stream; called where the host waits anyway).
static int tc_err_check(grim_context *h, const char *what) {
    if (!h->tc_err) return GRIM_OK;
    int v = 0;
    GRIM_CHECK_CUDA(cudaMemcpyAsync(&v, h->tc_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (v) {
        GRIM_CHECK_CUDA(cudaMemsetAsync(h->tc_err, 0, sizeof(int), h->stream));
        return grim_fail(GRIM_ERR_CUDA, std::string(what) + ": tensor-core pipeline wait timed out");
    }
    return GRIM_OK;
}

// A packed tensor-core operand (tile layout of tc_gemm.cuh): hi and lo arrays of
// rows_p x kp floats.
struct TcPacked {
    float *hi = nullptr, *lo = nullptr;
    int rows_p = 0, kp = 0;
};

static int tc_ws(grim_context *h, const char *name, int rows_p, int kp, TcPacked *out) {
    void *p = nullptr;
    GRIM_TRY(grim_workspace(h, name, 2 * (size_t)rows_p * kp * sizeof(float), &p));
    out->hi = (float *)p;
    out->lo = out->hi + (size_t)rows_p * kp;
    out->rows_p = rows_p;
    out->kp = kp;
    return GRIM_OK;
}

static inline int tc_rows_a(int M) { return ceil_div(2 * M, TC_BM) * TC_BM; }
static inline int tc_kp(int K) { return ceil_div(2 * K, TC_BK) * TC_BK; }
// Output-tile width: 128 columns for wide right-hand sides, 64 otherwise.
static inline int tc_bn(int N) { return N > 192 ? 128 : 64; }

static int tc_pack_a(grim_context *h, int M, int K, const float2 *A, int64_t lda, float sign, const TcPacked &P) {
    const int64_t chunks = (int64_t)P.rows_p * (P.kp / 4);
    k_tc_pack_a<<<ceil_div(chunks, 256), 256, 0, h->stream>>>(M, K, A, lda, P.hi, P.lo, P.rows_p, P.rows_p, 0, P.kp,
                                                              sign);
    GRIM_CHECK_LAUNCH_W(h, "k_tc_pack_a", 0.0, 8.0 * M * K + 32.0 * chunks);
    return GRIM_OK;
}

static int tc_pack_b(grim_context *h, int K, int N, const float2 *B, int64_t ldb, const TcPacked &P) {
    const int64_t chunks = (int64_t)P.rows_p * (P.kp / 4);
    k_tc_pack_b<<<ceil_div(chunks, 256), 256, 0, h->stream>>>(K, N, B, ldb, P.hi, P.lo, P.rows_p, P.kp);
    GRIM_CHECK_LAUNCH_W(h, "k_tc_pack_b", 0.0, 8.0 * K * N + 32.0 * chunks);
    return GRIM_OK;
}

template <int BN, int STAGES, bool STAGE_C>
static int tc_launch(grim_context *h, const TcPacked &A, const TcPacked &B, float2 *C, int64_t ldc, int M, int N,
                     int Kc, float alpha, int ow_lo, int ow_hi, int *err) {
    using Cfg = TcCfg<BN, STAGES, STAGE_C>;
    static PerDeviceOnce attr;
    if (attr.needed()) {
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_tc_gemm<BN, STAGES, STAGE_C>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM_BYTES));
        attr.mark();
    }
    dim3 grid(A.rows_p / TC_BM, ceil_div(N, BN));  // B.rows_p is the row stride of the packed B
    k_tc_gemm<BN, STAGES, STAGE_C><<<grid, TC_THREADS, Cfg::SMEM_BYTES, h->stream>>>(
        A.kp / TC_BK, A.hi, A.lo, A.rows_p, B.hi, B.lo, B.rows_p, (float *)C, 2 * ldc, 2 * M, N, alpha, 2 * ow_lo,
        2 * ow_hi, err);
    GRIM_CHECK_LAUNCH_W(h, BN == 128 ? "k_tc_gemm<128>" : "k_tc_gemm<64>", 8.0 * M * N * Kc,
                        8.0 * ((double)A.rows_p * A.kp * (B.rows_p / BN) + (double)B.rows_p * B.kp) + 16.0 * M * N);
    return GRIM_OK;
}

// Short inner dimensions (at most 8 K-tiles of 32 floats: the rank-64 factorization updates)
// spend most of a CTA's time in the epilogue: those launches stage C in shared memory during
// the main loop (two or three pipeline stages are enough for so few K-tiles).
#define TC_STAGE_C_MAX_KT 8

// C[M x N] = (complex rows in [ow_lo, ow_hi) ? 0 : C) + alpha * A B with packed A (2M real
// rows) and B (rows padded to bn); Kc is the complex inner dimension (for the flop count).
static int tc_gemm_packed(grim_context *h, int bn, const TcPacked &A, const TcPacked &B, float2 *C, int64_t ldc,
                          int M, int N, int Kc, float alpha, int ow_lo, int ow_hi) {
    if (M <= 0 || N <= 0) return GRIM_OK;
    if (A.kp != B.kp || B.rows_p % bn || A.rows_p % TC_BM || A.rows_p < 2 * M || B.rows_p < N)
        return grim_fail(GRIM_ERR_ARGUMENT, "tensor-core GEMM: packed operand shapes disagree");
    int *err;
    GRIM_TRY(tc_err_flag(h, &err));
    const bool stage_c = A.kp / TC_BK <= TC_STAGE_C_MAX_KT;
    if (bn == 128) {
        if (stage_c) return tc_launch<128, 2, true>(h, A, B, C, ldc, M, N, Kc, alpha, ow_lo, ow_hi, err);
        return tc_launch<128, 3, false>(h, A, B, C, ldc, M, N, Kc, alpha, ow_lo, ow_hi, err);
    }
    if (stage_c) return tc_launch<64, 3, true>(h, A, B, C, ldc, M, N, Kc, alpha, ow_lo, ow_hi, err);
    return tc_launch<64, 4, false>(h, A, B, C, ldc, M, N, Kc, alpha, ow_lo, ow_hi, err);
}

// C[MxN] = (overwrite ? 0 : C) + alpha A B[KxN] (complex64, column-major) on tcgen05 (split
// TF32), packing both operands.
static int tc_cgemm(grim_context *h, int M, int N, int K, const float2 *A, int64_t lda, const float2 *B, int64_t ldb,
                    float2 *C, int64_t ldc, float alpha, bool overwrite) {
    if (M <= 0 || N <= 0 || K <= 0) return GRIM_OK;
    const int bn = tc_bn(N), Kp = tc_kp(K);
    TcPacked pa, pb;
    GRIM_TRY(tc_ws(h, "tc_a", tc_rows_a(M), Kp, &pa));
    GRIM_TRY(tc_ws(h, "tc_b", ceil_div(N, bn) * bn, Kp, &pb));
    GRIM_TRY(tc_pack_a(h, M, K, A, lda, 1.f, pa));
    GRIM_TRY(tc_pack_b(h, K, N, B, ldb, pb));
    return tc_gemm_packed(h, bn, pa, pb, C, ldc, M, N, K, alpha, 0, overwrite ? M : 0);
}

// C[MxN] -= A B[KxN] on tcgen05.
static int tc_cgemm_sub(grim_context *h, int M, int N, int K, const float2 *A, int64_t lda, const float2 *B,
                        int64_t ldb, float2 *C, int64_t ldc) {
    return tc_cgemm(h, M, N, K, A, lda, B, ldb, C, ldc, -1.f, false);
}

// Trailing / solve updates C -= A B: tensor cores for complex64 (unless disabled), SIMT otherwise.
template <typename C>
static int gemm_sub(grim_context *h, int M, int N, int K, const C *A, int64_t lda, const C *B, int64_t ldb, C *Cm,
                    int64_t ldc) {
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (tc_enabled()) return tc_cgemm_sub(h, M, N, K, (const float2 *)A, lda, (const float2 *)B, ldb, (float2 *)Cm, ldc);
    }
    return gemm<C, C, C, C, true, true>(h, M, N, K, A, lda, B, ldb, Cm, ldc);
}

// Test entry: C -= A B for complex64 (use_tensor_cores 1: tcgen05 path, 0: SIMT path).
extern "C" int grim_cgemm_sub(grim_handle_t h, int M, int N, int K, const void *A, int64_t lda, const void *B,
                              int64_t ldb, void *Cm, int64_t ldc, int use_tensor_cores) {
    if (!h || M <= 0 || N <= 0 || K <= 0 || !A || !B || !Cm || lda < M || ldb < K || ldc < M)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_cgemm_sub: bad arguments");
    DeviceGuard g(h->device);
    if (use_tensor_cores) {
        GRIM_TRY(tc_cgemm_sub(h, M, N, K, (const float2 *)A, lda, (const float2 *)B, ldb, (float2 *)Cm, ldc));
        return tc_err_check(h, "grim_cgemm_sub");
    }
    return gemm<float2, float2, float2, float2, true, true>(h, M, N, K, (const float2 *)A, lda, (const float2 *)B, ldb,
                                                          (float2 *)Cm, ldc);
}

// ============================================================== getrf / getrs
template <typename C>
static int smem_opt_in() {
    static PerDeviceOnce done;
    if (!done.needed()) return GRIM_OK;
    const int tri = (NB * NBP + NB) * (int)sizeof(C);
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_panel_apply<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_panel_u_moves<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_tslu_finish<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_apply_moves<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         GEPP_MOVES_SMEM_MAX));
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_trsm_diag<C, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_trsm_diag<C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
    done.mark();
    return GRIM_OK;
}

static const char *kname(const char *base, size_t csize) {
    // kernel names for profiling, distinguished by precision
    static thread_local std::string s;
    s = std::string(base) + (csize == 16 ? "<c128>" : "<c64>");
    return s.c_str();
}

// Streams and events of the look-ahead (created once per handle).
static int lookahead_streams(grim_context *h, int nevents) {
    if (!h->chain) {
        int least = 0, greatest = 0;
        GRIM_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        GRIM_CHECK_CUDA(cudaStreamCreateWithPriority(&h->chain, cudaStreamNonBlocking, greatest));
        GRIM_CHECK_CUDA(cudaStreamCreateWithPriority(&h->bulk, cudaStreamNonBlocking, least));
    }
    while ((int)h->events.size() < nevents) {
        cudaEvent_t e;
        GRIM_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->events.push_back(e);
    }
    return GRIM_OK;
}

// Trailing update A22 -= L21 U12 split into the next panel's 64 columns ("narrow", on the
// current stream) and the rest ("wide", on `wide_stream`).  For complex64 both operands
// are packed once, into the buffer pair `slot`, and shared by the two tensor-core GEMMs.
// Packed operand buffers of one trailing update (double-buffered by panel parity); B rows
// padded so that a 128-wide tile starting at row 64 stays inside the buffer.
static int lu_packed(grim_context *h, int rest, int nbj, int slot, TcPacked *pa, TcPacked *pb) {
    const int Kp = tc_kp(nbj);
    GRIM_TRY(tc_ws(h, slot ? "lu_pa1" : "lu_pa0", tc_rows_a(rest), Kp, pa));
    GRIM_TRY(tc_ws(h, slot ? "lu_pb1" : "lu_pb0", ceil_div(rest + NB, 128) * 128, Kp, pb));
    return GRIM_OK;
}

// prepacked: the panel solve already wrote both operands into the slot's buffers.
template <typename C>
static int trailing_update(grim_context *h, int rest, int nbj, const C *L21, const C *U12, C *A22, int64_t lda,
                           cudaStream_t wide_stream, cudaEvent_t packed, int slot, bool prepacked = false) {
    const int nn = std::min(NB, rest), nw = rest - nn;
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (tc_enabled()) {
            TcPacked pa, pb;
            GRIM_TRY(lu_packed(h, rest, nbj, slot, &pa, &pb));
            if (!prepacked) {
                GRIM_TRY(tc_pack_a(h, rest, nbj, (const float2 *)L21, lda, 1.f, pa));
                GRIM_TRY(tc_pack_b(h, nbj, rest, (const float2 *)U12, lda, pb));
            }
            GRIM_TRY(tc_gemm_packed(h, 64, pa, pb, (float2 *)A22, lda, rest, nn, nbj, -1.f, 0, 0));
            if (nw > 0) {
                GRIM_CHECK_CUDA(cudaEventRecord(packed, h->stream));
                GRIM_CHECK_CUDA(cudaStreamWaitEvent(wide_stream, packed, 0));
                const cudaStream_t keep = h->stream;
                h->stream = wide_stream;
                TcPacked pw = pb;
                pw.hi += (size_t)NB * 32;
                pw.lo += (size_t)NB * 32;
                const int bn = tc_bn(nw);
                int s = tc_gemm_packed(h, bn, pa, pw, (float2 *)(A22 + (int64_t)nn * lda), lda, rest, nw, nbj, -1.f, 0,
                                       0);
                h->stream = keep;
                GRIM_TRY(s);
            }
            return GRIM_OK;
        }
    }
    GRIM_TRY((gemm<C, C, C, C, true, true>(h, rest, nn, nbj, L21, lda, U12, lda, A22, lda)));
    if (nw > 0) {
        GRIM_CHECK_CUDA(cudaEventRecord(packed, h->stream));
        GRIM_CHECK_CUDA(cudaStreamWaitEvent(wide_stream, packed, 0));
        const cudaStream_t keep = h->stream;
        h->stream = wide_stream;
        int s = gemm<C, C, C, C, true, true>(h, rest, nw, nbj, L21, lda, U12 + (int64_t)nn * lda, lda,
                                             A22 + (int64_t)nn * lda, lda);
        h->stream = keep;
        GRIM_TRY(s);
    }
    return GRIM_OK;
}

// Rows per cluster CTA of the partial-pivoting panel: a panel of m rows takes the smallest
// power-of-two cluster (at most 16 CTAs) that keeps each CTA's rows within this target
// (GRIM_GEPP_ROWS overrides), so that short panels pay for few cluster barriers.
static int gepp_rows_target(size_t csize) {
    static const int env = [] {
        const char *e = getenv("GRIM_GEPP_ROWS");
        return e ? atoi(e) : 0;
    }();
    if (env >= 32) return env;
    return 128;
}

// Register-resident panel rows (k_panel_gepp_reg) for panels of at most 16 x GEPPR_ROWS rows;
// GRIM_GEPP_REG=0 keeps every panel on the shared-memory kernel.
static bool gepp_reg_enabled() {
    static const bool on = [] {
        const char *e = getenv("GRIM_GEPP_REG");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

// Loop-resident partial-pivoting panel (k_panel_gepp_loop) for panels of at most
// 16 x GEPPL_ROWS rows; GRIM_GEPP_LOOP=0 keeps them on the unrolled register kernel.
static bool gepp_loop_enabled() {
    static const bool on = [] {
        const char *e = getenv("GRIM_GEPP_LOOP");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

// GRIM_GEPP_PUSH=1: candidate rows pushed into every CTA before the cluster barrier
// (k_panel_gepp_loop PUSH).  Off by default: measured on the 2048-row panels it takes 132 us
// against 119 us for reading only the winner's row through distributed shared memory after
// the barrier (the pushes move 16 rows per CTA per column where the read moves one).
static bool gepp_push_enabled() {
    static const bool on = [] {
        const char *e = getenv("GRIM_GEPP_PUSH");
        return e && atoi(e) == 1;
    }();
    return on;
}

// Partial-pivoting factorization of the panel (j, nbj) of A on one thread-block cluster.
template <typename C>
static int gepp_launch(grim_context *h, int n, C *A, int64_t lda, int j, int nbj, int *ipiv, int *d_info,
                       int *swapped, int *moves, PanelPack pk) {
    const int m = n - j;
    if (gepp_loop_enabled() && m <= 16 * GEPPL_ROWS) {
        const int cs = std::max(1, ceil_div(m, GEPPL_ROWS));
        const int rpc = ceil_div(m, cs);
        const bool push = gepp_push_enabled();
        const size_t smem = ((size_t)NB * GEPPL_ROWS + (push ? (size_t)2 * 16 * 2 * NB : 0)) * sizeof(C);
        auto kern = push ? k_panel_gepp_loop<C, true> : k_panel_gepp_loop<C, false>;
        static PerDeviceOnce attr_loop;
        if (attr_loop.needed()) {
            for (auto kf : {k_panel_gepp_loop<C, true>, k_panel_gepp_loop<C, false>}) {
                const size_t sm = ((size_t)NB * GEPPL_ROWS + (size_t)2 * 16 * 2 * NB) * sizeof(C);
                GRIM_CHECK_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                GRIM_CHECK_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            }
            attr_loop.mark();
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(GEPPL_THREADS);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = h->stream;
        cudaLaunchAttribute la[1];
        la[0].id = cudaLaunchAttributeClusterDimension;
        la[0].val.clusterDim.x = cs;
        la[0].val.clusterDim.y = 1;
        la[0].val.clusterDim.z = 1;
        cfg.attrs = la;
        cfg.numAttrs = 1;
        GRIM_CHECK_CUDA(cudaLaunchKernelEx(&cfg, kern, n, A, lda, j, nbj, rpc, ipiv, d_info, swapped, moves, pk));
        return grim_launch_status(h, kname("k_panel_gepp_loop", sizeof(C)), 8.0 * m * nbj * nbj / 2.0, 0);
    }
    if (gepp_reg_enabled() && m <= 16 * GEPPR_ROWS) {
        // rows in registers: the fewest CTAs of at most GEPPR_ROWS rows each
        const int cs = std::max(1, ceil_div(m, GEPPR_ROWS));
        const int rpc = ceil_div(m, cs);
        static PerDeviceOnce attr_reg;
        if (attr_reg.needed()) {
            GRIM_CHECK_CUDA(
                cudaFuncSetAttribute(k_panel_gepp_reg<C>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            attr_reg.mark();
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(GEPP_THREADS);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = h->stream;
        cudaLaunchAttribute la[1];
        la[0].id = cudaLaunchAttributeClusterDimension;
        la[0].val.clusterDim.x = cs;
        la[0].val.clusterDim.y = 1;
        la[0].val.clusterDim.z = 1;
        cfg.attrs = la;
        cfg.numAttrs = 1;
        GRIM_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_panel_gepp_reg<C>, n, A, lda, j, nbj, rpc, ipiv, d_info, swapped,
                                           moves, pk));
        return grim_launch_status(h, kname("k_panel_gepp_reg", sizeof(C)), 8.0 * m * nbj * nbj / 2.0, 0);
    }
    const int target = gepp_rows_target(sizeof(C));
    int cs = 1;
    while (cs < 16 && ceil_div(m, cs) > target) cs <<= 1;
    const int rpc = ceil_div(m, cs);
    const size_t fixed = gepp_fixed_smem<C>();
    const size_t cap = (size_t)227 * 1024 - 1024 - fixed;
    const int rows_smem = std::min(rpc, (int)(cap / (GEPP_LDR * sizeof(C))));
    const size_t smem = fixed + (size_t)rows_smem * GEPP_LDR * sizeof(C);
    C *gs = nullptr;
    if (rpc > rows_smem) {
        void *p = nullptr;
        GRIM_TRY(grim_workspace(h, sizeof(C) == 16 ? "gepp_scratch64" : "gepp_scratch32",
                                (size_t)cs * (rpc - rows_smem) * NB * sizeof(C), &p));
        gs = (C *)p;
    }
    static PerDeviceOnce attr;
    if (attr.needed()) {
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_panel_gepp<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             227 * 1024 - 1024));
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_panel_gepp<C>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        attr.mark();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(GEPP_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cudaLaunchAttribute la[1];
    la[0].id = cudaLaunchAttributeClusterDimension;
    la[0].val.clusterDim.x = cs;
    la[0].val.clusterDim.y = 1;
    la[0].val.clusterDim.z = 1;
    cfg.attrs = la;
    cfg.numAttrs = 1;
    GRIM_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_panel_gepp<C>, n, A, lda, j, nbj, rpc, rows_smem, gs, ipiv, d_info,
                                       swapped, moves, pk));
    return grim_launch_status(h, kname("k_panel_gepp", sizeof(C)), 8.0 * m * nbj * nbj / 2.0, 0);
}

// Tournament-pivoting panel (tslu.cuh): the selection tree, then L21 and the row moves.
// ws: the factorization's tournament workspace (TsluWs, sized for its n).
struct TsluWs {
    int *cand = nullptr, *ccount = nullptr, *arrive = nullptr, *winners = nullptr;
    void *top = nullptr;
    int gmax = 0;  // CTAs of the first panel: arrive holds 2 gmax + 32 counters per panel
};

template <typename C>
static int tslu_workspace(grim_context *h, int n, TsluWs *ws) {
    const int npan = ceil_div(n, NB);
    ws->gmax = ceil_div(n, TSLU_ROWS);
    void *p = nullptr;
    // nodes of one tree: sum over levels of ceil(g / 2^l) <= 2 g + log2(g)
    const size_t nodes = (size_t)2 * ws->gmax + 32;
    GRIM_TRY(grim_workspace(h, "tslu_nodes", nodes * (NB + 1) * sizeof(int) + NB * sizeof(int), &p));
    ws->cand = (int *)p;
    ws->ccount = ws->cand + nodes * NB;
    ws->winners = ws->ccount + nodes;
    GRIM_TRY(grim_workspace(h, sizeof(C) == 16 ? "tslu_top64" : "tslu_top32", (size_t)NB * NB * sizeof(C), &p));
    ws->top = p;
    GRIM_TRY(grim_workspace(h, "tslu_arrive", (size_t)npan * nodes * sizeof(int), &p));
    ws->arrive = (int *)p;
    GRIM_CHECK_CUDA(cudaMemsetAsync(ws->arrive, 0, (size_t)npan * nodes * sizeof(int), h->stream));
    return GRIM_OK;
}

template <typename C>
static int tslu_launch(grim_context *h, int n, C *A, int64_t lda, int p, int j, int nbj, int *ipiv, int *d_info,
                       int *swapped, int *moves, PanelPack pk, const TsluWs &ws) {
    const int m = n - j;
    const int g = ceil_div(m, TSLU_ROWS);
    int *arrive = ws.arrive + (size_t)p * (2 * ws.gmax + 32);
    k_tslu_tree<C><<<g, TSLU_THREADS, 0, h->stream>>>(n, A, lda, j, nbj, ws.cand, ws.ccount, arrive, (C *)ws.top,
                                                     ws.winners, ipiv, d_info, swapped, moves);
    GRIM_TRY(grim_launch_status(h, kname("k_tslu_tree", sizeof(C)), 8.0 * m * nbj * nbj / 2.0, 0));
    const size_t tri = (size_t)(NB * NBP + NB) * sizeof(C);
    k_tslu_finish<C><<<g, 256, tri, h->stream>>>(n, A, lda, j, nbj, (const C *)ws.top, ws.winners, moves, pk);
    return grim_launch_status(h, kname("k_tslu_finish", sizeof(C)), 8.0 * m * nbj * nbj / 2.0, 0);
}

// Device flag layout for one factorization: [0] info, [1] pivoted panels, then per panel
// cert[npan], swapped[npan], counter[npan].
//
// Look-ahead: the panel chain (diagonal block, panel solve, the next panel's 64-column
// update) runs on a high-priority stream, the rest of each trailing update on a
// low-priority one, so that the diagonal block of panel p+1 is factored while the wide
// update of panel p is still running; panel p+1's solve waits for that update (its U12
// reads the updated columns).  With per-launch profiling on, everything runs on the
// handle's stream in order.
// defer: return without reading the info / pivoted-panel flags on the host (no host
// synchronisation: the caller queues its solves behind the factorization and reads them
// later with getrf_read_flags); *info_host is then 0.
template <typename C>
static int getrf_impl(grim_context *h, int n, C *A, int64_t lda, int *ipiv, int *info_host, bool defer = false) {
    if (!h || n <= 0 || !A || lda < n || !ipiv) return grim_fail(GRIM_ERR_ARGUMENT, "getrf: bad arguments");
    DeviceGuard g(h->device);
    GRIM_TRY(smem_opt_in<C>());
    const int npan = ceil_div(n, NB);
    void *p_bc = nullptr, *p_br = nullptr, *p_flags = nullptr;
    GRIM_TRY(grim_workspace(h, "lu_backup_col", (size_t)n * NB * sizeof(C), &p_bc));
    GRIM_TRY(grim_workspace(h, "lu_backup_row", (size_t)n * NB * sizeof(C), &p_br));
    GRIM_TRY(grim_workspace(h, "lu_flags", (size_t)(2 + 3 * npan) * sizeof(int), &p_flags));
    C *bcol = (C *)p_bc, *brow = (C *)p_br;
    int *flags = (int *)p_flags;
    int *d_info = flags, *d_pivoted = flags + 1, *cert = flags + 2, *swapped = cert + npan, *counter = swapped + npan;
    GRIM_CHECK_CUDA(cudaMemsetAsync(flags, 0, (size_t)(2 + 3 * npan) * sizeof(int), h->stream));
    const size_t tri = (size_t)(NB * NBP + NB) * sizeof(C);
    const bool split = !h->profiling;
    const cudaStream_t caller = h->stream;
    cudaStream_t wide = caller;
    // events: [0] start, [1] end, then per panel "packed" (2 + p) and "wide done" (2 + npan + p)
    if (split) {
        GRIM_TRY(lookahead_streams(h, 2 + 2 * npan));
        GRIM_CHECK_CUDA(cudaEventRecord(h->events[0], caller));
        GRIM_CHECK_CUDA(cudaStreamWaitEvent(h->chain, h->events[0], 0));
        GRIM_CHECK_CUDA(cudaStreamWaitEvent(h->bulk, h->events[0], 0));
        h->stream = h->chain;
        wide = h->bulk;
    } else {
        GRIM_TRY(lookahead_streams(h, 2 + 2 * npan));
    }
    int status = GRIM_OK;
    bool wide_pending = false;
    int *moves = nullptr;
    const bool tournament = h->pivot_mode == GRIM_PIVOT_TOURNAMENT;
    TsluWs tws;
    if (h->pivot_mode == GRIM_PIVOT_PARTIAL || tournament) {
        void *pm = nullptr;
        GRIM_TRY(grim_workspace(h, "gepp_moves", (1 + 2 * GEPP_MAX_MOVES) * sizeof(int), &pm));
        moves = (int *)pm;
        if (tournament) GRIM_TRY(tslu_workspace<C>(h, n, &tws));
    }
    for (int p = 0; p < npan && status == GRIM_OK && moves; ++p) {
        // partial pivoting: the panel on a cluster, then the trailing columns' row moves and
        // U12, then the trailing update (the same look-ahead as below)
        const int j = p * NB, nbj = std::min(NB, n - j);
        const int rest = n - j - nbj;
        PanelPack pk;
        const bool prepack = sizeof(C) == sizeof(float2) && tc_enabled() && nbj == NB && rest > 0;
        if (prepack) {
            TcPacked pa, pb;
            status = lu_packed(h, rest, nbj, p & 1, &pa, &pb);
            if (status != GRIM_OK) break;
            pk.a_hi = pa.hi;
            pk.a_lo = pa.lo;
            pk.a_rows = pa.rows_p;
            pk.b_hi = pb.hi;
            pk.b_lo = pb.lo;
            pk.b_rows = pb.rows_p;
        }
        status = tournament ? tslu_launch<C>(h, n, A, lda, p, j, nbj, ipiv, d_info, swapped + p, moves, pk, tws)
                            : gepp_launch<C>(h, n, A, lda, j, nbj, ipiv, d_info, swapped + p, moves, pk);
        if (status != GRIM_OK) break;
        if (wide_pending) {
            GRIM_CHECK_CUDA(cudaStreamWaitEvent(h->stream, h->events[2 + npan + p - 1], 0));
            wide_pending = false;
        }
        if (rest > 0) {
            k_panel_u_moves<C><<<ceil_div(rest, UMOVES_THREADS / 4), UMOVES_THREADS, tri, h->stream>>>(n, A, lda, j,
                                                                                                   nbj, moves, pk);
            status = grim_launch_status(h, kname("k_panel_u_moves", sizeof(C)), 8.0 * rest * nbj * nbj / 2.0, 0);
            if (status != GRIM_OK) break;
            status = trailing_update<C>(h, rest, nbj, A + (int64_t)j * lda + j + nbj, A + (int64_t)(j + nbj) * lda + j,
                                        A + (int64_t)(j + nbj) * lda + j + nbj, lda, wide, h->events[2 + p], p & 1,
                                        prepack);
            if (status != GRIM_OK) break;
            if (rest > NB && split) {
                status = grim_cuda_status(cudaEventRecord(h->events[2 + npan + p], wide), "cudaEventRecord");
                wide_pending = status == GRIM_OK;
            }
        }
    }
    for (int p = 0; p < npan && status == GRIM_OK && !moves; ++p) {
        const int j = p * NB, nbj = std::min(NB, n - j);
        k_diag_lu<C><<<1, 256, 0, h->stream>>>(n, A, lda, j, nbj, bcol, cert + p, ipiv);
        status = grim_launch_status(h, kname("k_diag_lu", sizeof(C)), 8.0 * nbj * nbj * nbj / 3.0, 0);
        if (status != GRIM_OK) break;
        if (wide_pending) {
            GRIM_CHECK_CUDA(cudaStreamWaitEvent(h->stream, h->events[2 + npan + p - 1], 0));
            wide_pending = false;
        }
        const int rest = n - j - nbj;
        if (rest > 0) {
            const int nL = ceil_div(rest, NB), nU = nL;
            // complex64 on tensor cores: the panel solve writes the update's packed operands
            PanelPack pk;
            const bool prepack = sizeof(C) == sizeof(float2) && tc_enabled() && nbj == NB;
            if (prepack) {
                TcPacked pa, pb;
                status = lu_packed(h, rest, nbj, p & 1, &pa, &pb);
                if (status != GRIM_OK) break;
                pk.a_hi = pa.hi;
                pk.a_lo = pa.lo;
                pk.a_rows = pa.rows_p;
                pk.b_hi = pb.hi;
                pk.b_lo = pb.lo;
                pk.b_rows = pb.rows_p;
            }
            k_panel_apply<C><<<nL + nU, 256, tri, h->stream>>>(n, A, lda, j, nbj, nL, bcol, brow, cert + p,
                                                               counter + p, swapped + p, ipiv, d_info, d_pivoted, pk,
                                                               h->pivot_mode == GRIM_PIVOT_STATIC);
            status = grim_launch_status(h, kname("k_panel_apply", sizeof(C)), 8.0 * 2 * rest * nbj * nbj, 0);
            if (status != GRIM_OK) break;
            status = trailing_update<C>(h, rest, nbj, A + (int64_t)j * lda + j + nbj, A + (int64_t)(j + nbj) * lda + j,
                                        A + (int64_t)(j + nbj) * lda + j + nbj, lda, wide, h->events[2 + p], p & 1,
                                        prepack);
            if (status != GRIM_OK) break;
            if (rest > NB && split) {
                status = grim_cuda_status(cudaEventRecord(h->events[2 + npan + p], wide), "cudaEventRecord");
                wide_pending = status == GRIM_OK;
            }
        } else {
            k_panel_last<C><<<1, 256, 0, h->stream>>>(n, A, lda, j, nbj, bcol, cert + p, swapped + p, ipiv, d_info,
                                                      d_pivoted, h->pivot_mode == GRIM_PIVOT_STATIC);
            status = grim_launch_status(h, kname("k_panel_last", sizeof(C)), 0, 0);
        }
    }
    if (status == GRIM_OK && moves && (size_t)n * sizeof(C) <= GEPP_MOVES_SMEM_MAX && n > NB) {
        // partial pivoting: every panel's row moves, then each factored column takes those of
        // the panels after it (one CTA per column, in shared memory)
        void *pm = nullptr;
        status = grim_workspace(h, "lu_moves_all", (size_t)npan * GEPP_MOVES_STRIDE * sizeof(int), &pm);
        if (status == GRIM_OK) {
            k_ipiv_moves<<<ceil_div(npan, 4), 128, 0, h->stream>>>(n, ipiv, (int *)pm);
            status = grim_launch_status(h, "k_ipiv_moves", 0, 0);
        }
        if (status == GRIM_OK) {
            const int ncols = (npan - 1) * NB;
            k_apply_moves<C><<<ncols, 256, (size_t)n * sizeof(C), h->stream>>>(n, A, lda, 0, 1, (const int *)pm,
                                                                                nullptr);
            status = grim_launch_status(h, kname("k_apply_moves_left", sizeof(C)), 0, 0);
        }
    } else if (status == GRIM_OK) {
        k_laswp_left<C><<<ceil_div(n, 128), 128, 0, h->stream>>>(n, A, lda, NB, swapped, ipiv);
        status = grim_launch_status(h, kname("k_laswp_left", sizeof(C)), 0, 0);
    }
    if (split) {
        // the caller's stream waits for both streams, whatever happened above
        cudaEventRecord(h->events[1], h->bulk);
        cudaStreamWaitEvent(h->chain, h->events[1], 0);
        cudaEventRecord(h->events[1], h->chain);
        cudaStreamWaitEvent(caller, h->events[1], 0);
        h->stream = caller;
    }
    GRIM_TRY(status);
    if (defer) {
        if (info_host) *info_host = 0;
        return GRIM_OK;
    }
    int hostf[2] = {0, 0};
    GRIM_CHECK_CUDA(cudaMemcpyAsync(hostf, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (sizeof(C) == sizeof(float2)) GRIM_TRY(tc_err_check(h, "getrf"));
    if (info_host) *info_host = hostf[0];
    h->last.pivoted_panels = hostf[1];
    h->last.info = hostf[0];
    return GRIM_OK;
}

// The info and pivoted-panel counts of the last deferred getrf_impl on this handle.
static int getrf_read_flags(grim_context *h, int *info, int *pivoted) {
    void *p_flags = nullptr;
    GRIM_TRY(grim_workspace(h, "lu_flags", 2 * sizeof(int), &p_flags));
    int hostf[2] = {0, 0};
    GRIM_CHECK_CUDA(cudaMemcpyAsync(hostf, p_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    *info = hostf[0];
    *pivoted = hostf[1];
    return GRIM_OK;
}

// getrs: interchanges (skipped when ipiv is the identity), then per 64-row block an
// in-place diagonal triangular solve and a GEMM update of the remaining rows.
static int rs_moves(grim_context *h, int n, int **out) {
    void *p = nullptr;
    GRIM_TRY(grim_workspace(h, "rs_moves", (size_t)ceil_div(n, NB) * GEPP_MOVES_STRIDE * sizeof(int), &p));
    *out = (int *)p;
    return GRIM_OK;
}

template <typename C>
static int getrs_prepare(grim_context *h, int n, const int *ipiv, int **ident_out) {
    void *p_id = nullptr;
    GRIM_TRY(grim_workspace(h, sizeof(C) == 16 ? "rs_ident64" : "rs_ident32", sizeof(int), &p_id));
    int *ident = (int *)p_id;
    GRIM_CHECK_CUDA(cudaMemsetAsync(ident, 0xff, sizeof(int), h->stream));
    k_ipiv_identity<<<ceil_div(n, 256), 256, 0, h->stream>>>(n, ipiv, ident);
    GRIM_CHECK_LAUNCH(h, "k_ipiv_identity");
    if ((size_t)n * sizeof(C) <= GEPP_MOVES_SMEM_MAX) {
        // the row moves of every panel, for the right-hand sides' interchanges
        int *mv = nullptr;
        GRIM_TRY(rs_moves(h, n, &mv));
        k_ipiv_moves<<<ceil_div(ceil_div(n, NB), 4), 128, 0, h->stream>>>(n, ipiv, mv);
        GRIM_CHECK_LAUNCH(h, "k_ipiv_moves");
    }
    *ident_out = ident;
    return GRIM_OK;
}

// Right-hand-side interchanges of getrs: the panels' row moves applied in shared memory, one
// CTA per column (the rows moves of getrs_prepare), or LAPACK's sequential swaps when a
// column does not fit.
template <typename C>
static int rhs_interchanges(grim_context *h, int n, int nrhs, C *B, int64_t ldb, const int *ipiv, const int *ident) {
    if ((size_t)n * sizeof(C) <= GEPP_MOVES_SMEM_MAX) {
        int *mv = nullptr;
        GRIM_TRY(rs_moves(h, n, &mv));
        k_apply_moves<C><<<nrhs, 256, (size_t)n * sizeof(C), h->stream>>>(n, B, ldb, 0, 0, mv, ident);
        GRIM_CHECK_LAUNCH(h, kname("k_apply_moves_rhs", sizeof(C)));
        return GRIM_OK;
    }
    k_laswp_rhs<C><<<ceil_div(nrhs, 128), 128, 0, h->stream>>>(n, nrhs, B, ldb, ipiv, ident);
    GRIM_CHECK_LAUNCH(h, kname("k_laswp_rhs", sizeof(C)));
    return GRIM_OK;
}

template <typename C>
static int getrs_apply(grim_context *h, int n, int nrhs, const C *LU, int64_t lda, const int *ipiv, const int *ident,
                       C *B, int64_t ldb) {
    const int npan = ceil_div(n, NB);
    const size_t tri = (size_t)(NB * NBP + NB) * sizeof(C);
    GRIM_TRY(rhs_interchanges<C>(h, n, nrhs, B, ldb, ipiv, ident));
    const int ctiles = ceil_div(nrhs, TRSM_COLS);
    for (int p = 0; p < npan; ++p) {
        const int j = p * NB, nbj = std::min(NB, n - j);
        k_trsm_diag<C, false><<<ctiles, 4 * TRSM_COLS, tri, h->stream>>>(nrhs, LU, lda, B, ldb, j, nbj, 0, 0);
        GRIM_CHECK_LAUNCH_W(h, kname("k_trsm_diag", sizeof(C)), 4.0 * nbj * nbj * nrhs, 0);
        const int below = n - j - nbj;
        if (below > 0)
            GRIM_TRY((gemm_sub<C>(h, below, nrhs, nbj, LU + (int64_t)j * lda + j + nbj, lda, B + j, ldb,
                                                  B + j + nbj, ldb)));
    }
    for (int p = npan - 1; p >= 0; --p) {
        const int j = p * NB, nbj = std::min(NB, n - j);
        k_trsm_diag<C, true><<<ctiles, 4 * TRSM_COLS, tri, h->stream>>>(nrhs, LU, lda, B, ldb, j, nbj, 0, 0);
        GRIM_CHECK_LAUNCH_W(h, kname("k_trsm_diag", sizeof(C)), 4.0 * nbj * nbj * nrhs, 0);
        if (j > 0)
            GRIM_TRY((gemm_sub<C>(h, j, nrhs, nbj, LU + (int64_t)j * lda, lda, B + j, ldb, B, ldb)));
    }
    return GRIM_OK;
}

template <typename C>
static int getrs_impl(grim_context *h, int n, int nrhs, const C *LU, int64_t lda, const int *ipiv, C *B, int64_t ldb) {
    if (!h || n <= 0 || nrhs <= 0 || !LU || !ipiv || !B || lda < n || ldb < n)
        return grim_fail(GRIM_ERR_ARGUMENT, "getrs: bad arguments");
    DeviceGuard g(h->device);
    GRIM_TRY(smem_opt_in<C>());
    int *ident;
    GRIM_TRY(getrs_prepare<C>(h, n, ipiv, &ident));
    return getrs_apply<C>(h, n, nrhs, LU, lda, ipiv, ident, B, ldb);
}

// ------------------------------------------------ complex64 getrs on packed block panels
// For many right-hand sides the two triangular solves run in nb-row blocks, each block
// one tensor-core GEMM with a panel formed once per factorization:
//   forward  (L unit lower), block i at rows J..J+nb:  PL_i = [Linv_ii; -L_below,i Linv_ii]
//            B[J:n] = [0; B[J+nb:n]] + PL_i B[J:J+nb]
//   backward (U upper),      block i:                  PU_i = [-U_above,i Uinv_ii; Uinv_ii]
//            B[0:J+nb] = [B[0:J]; 0] + PU_i B[J:J+nb]
// The inverses of all diagonal blocks are formed together (batched over blocks: the
// 64-row triangular solves of k_trsm_diag on identity columns, then SIMT updates inside
// each block), the off-diagonal parts by one tensor-core GEMM per block, and both are
// packed (split TF32, tile layout) and kept for every solve of a refinement loop.  The
// block solve multiplies by the inverse of a triangular diagonal block instead of
// substituting; its rounding is that of an FP32 GEMM, and the FP64 refinement that
// consumes these solves removes it.
// Block height: 512 rows for large, wide solves (fewer, longer GEMMs), 256 otherwise (a
// cheaper panel build when it is amortised over fewer right-hand sides).
#define GS_NB_MAX 512
static inline int gs_block(int n, int nrhs) { return (n >= 2048 && nrhs >= 512) ? 512 : 256; }

struct GsPanels {
    int n = 0, nblk = 0, nb = 256;
    std::vector<TcPacked> L, U;
};

// T_b (bd x bd, leading dim ldt, batch stride sT) = inverse of the unit lower (upper =
// false) or upper diagonal block of LU at (J0 + b nb) for b < count, by 64-row
// substitution steps (used for a partial last block).
static int gs_invert_blocks(grim_context *h, const float2 *LU, int64_t lda, int J0, int count, int bd, float2 *T,
                            int64_t ldt, int64_t sT, bool upper, int nb) {
    const size_t tri = (size_t)(NB * NBP + NB) * sizeof(float2);
    const int64_t sLU = (int64_t)nb * (lda + 1);
    const float2 *D = LU + (int64_t)J0 * lda + J0;
    k_set_unit<float2><<<dim3(ceil_div(bd, 256), bd, count), 256, 0, h->stream>>>(bd, bd, T, ldt, 0, sT);
    GRIM_CHECK_LAUNCH(h, "k_set_unit");
    const int nsub = ceil_div(bd, NB);
    for (int q = 0; q < nsub; ++q) {
        const int s = upper ? nsub - 1 - q : q, js = s * NB, nbs = std::min(NB, bd - js);
        dim3 tg(ceil_div(bd, TRSM_COLS), count);
        if (upper)
            k_trsm_diag<float2, true><<<tg, 4 * TRSM_COLS, tri, h->stream>>>(bd, D, lda, T, ldt, js, nbs, sLU, sT);
        else
            k_trsm_diag<float2, false><<<tg, 4 * TRSM_COLS, tri, h->stream>>>(bd, D, lda, T, ldt, js, nbs, sLU, sT);
        GRIM_CHECK_LAUNCH_W(h, "k_trsm_diag<c64>", 4.0 * nbs * nbs * bd * count, 0);
        // rows of the block still to solve: below the strip (lower) or above it (upper)
        const int M = upper ? js : bd - js - nbs;
        if (M <= 0) continue;
        const float2 *Ab = upper ? D + (int64_t)js * lda : D + (int64_t)js * lda + js + nbs;
        float2 *Cb = upper ? T : T + js + nbs;
        dim3 grid(ceil_div(M, RT_BM), ceil_div(bd, RT_BN), count);
        k_gemm_rt<float2, float2, float2, float2, true, true><<<grid, RT_THREADS, 0, h->stream>>>(
            M, bd, nbs, Ab, lda, T + js, ldt, Cb, ldt, sLU, sT, sT);
        GRIM_CHECK_LAUNCH_W(h, "k_gemm_rt<f32>", 8.0 * M * bd * nbs * count, 0);
    }
    return GRIM_OK;
}

// Inverses of the diagonal nb-blocks of the first `rows` rows (a multiple of nb) of the
// unit lower (upper = false) or upper factor, into the same positions of T (leading dim
// ldt; T zeroed outside the blocks), by recursive doubling: the 64 x 64 diagonal blocks
// are inverted by one batched substitution launch, then, for s = 64, 128, ..., nb / 2,
// every 2s-block [A 0; C D] (lower) gets its off-diagonal part -D^-1 (C A^-1), or
// [A B; 0 D] (upper) gets -A^-1 (B D^-1), by two batched GEMMs over all 2s-blocks.
static int gs_invert_recursive(grim_context *h, const float2 *LU, int64_t lda, int rows, int nb, float2 *T,
                               int64_t ldt, float2 *TW, bool upper) {
    const size_t tri = (size_t)(NB * NBP + NB) * sizeof(float2);
    const int nq = rows / NB;
    GRIM_CHECK_CUDA(cudaMemset2DAsync(T, ldt * sizeof(float2), 0, rows * sizeof(float2), rows, h->stream));
    k_set_unit<float2><<<dim3(1, NB, nq), NB, 0, h->stream>>>(NB, NB, T, ldt, 0, (int64_t)NB * (ldt + 1));
    GRIM_CHECK_LAUNCH(h, "k_set_unit");
    dim3 tg(NB / TRSM_COLS, nq);
    if (upper)
        k_trsm_diag<float2, true><<<tg, 4 * TRSM_COLS, tri, h->stream>>>(NB, LU, lda, T, ldt, 0, NB,
                                                                         (int64_t)NB * (lda + 1),
                                                                         (int64_t)NB * (ldt + 1));
    else
        k_trsm_diag<float2, false><<<tg, 4 * TRSM_COLS, tri, h->stream>>>(NB, LU, lda, T, ldt, 0, NB,
                                                                          (int64_t)NB * (lda + 1),
                                                                          (int64_t)NB * (ldt + 1));
    GRIM_CHECK_LAUNCH_W(h, "k_trsm_diag<c64>", 4.0 * NB * NB * NB * nq, 0);
    for (int s = NB; s < nb; s *= 2) {
        const int count = rows / (2 * s);
        const int64_t sLU = (int64_t)2 * s * (lda + 1), sT = (int64_t)2 * s * (ldt + 1), sW = (int64_t)s * s;
        dim3 grid(ceil_div(s, RT_BM), ceil_div(s, RT_BN), count);
        if (!upper) {
            // W = C A^-1;  X = -D^-1 W  (C = L[o+s:o+2s, o:o+s], X at T[o+s:, o:])
            k_gemm_rt<float2, float2, float2, float2, false, false><<<grid, RT_THREADS, 0, h->stream>>>(
                s, s, s, LU + s, lda, T, ldt, TW, s, sLU, sT, sW);
            GRIM_CHECK_LAUNCH_W(h, "k_gemm_rt<f32>", 8.0 * s * s * s * count, 0);
            k_gemm_rt<float2, float2, float2, float2, true, false><<<grid, RT_THREADS, 0, h->stream>>>(
                s, s, s, T + (int64_t)s * (ldt + 1), ldt, TW, s, T + s, ldt, sT, sW, sT);
            GRIM_CHECK_LAUNCH_W(h, "k_gemm_rt<f32>", 8.0 * s * s * s * count, 0);
        } else {
            // W = B D^-1;  X = -A^-1 W  (B = U[o:o+s, o+s:o+2s], X at T[o:, o+s:])
            k_gemm_rt<float2, float2, float2, float2, false, false><<<grid, RT_THREADS, 0, h->stream>>>(
                s, s, s, LU + (int64_t)s * lda, lda, T + (int64_t)s * (ldt + 1), ldt, TW, s, sLU, sT, sW);
            GRIM_CHECK_LAUNCH_W(h, "k_gemm_rt<f32>", 8.0 * s * s * s * count, 0);
            k_gemm_rt<float2, float2, float2, float2, true, false><<<grid, RT_THREADS, 0, h->stream>>>(
                s, s, s, T, ldt, TW, s, T + (int64_t)s * ldt, ldt, sT, sW, sT);
            GRIM_CHECK_LAUNCH_W(h, "k_gemm_rt<f32>", 8.0 * s * s * s * count, 0);
        }
    }
    return GRIM_OK;
}

static int gs_build(grim_context *h, int n, const float2 *LU, int64_t lda, int nb, GsPanels *P) {
    const int nblk = ceil_div(n, nb), nfull = n / nb;
    size_t floats_l = 0, floats_u = 0;
    for (int i = 0; i < nblk; ++i) {
        const int J = i * nb, nbj = std::min(nb, n - J);
        floats_l += 2 * (size_t)tc_rows_a(n - J) * tc_kp(nbj);
        floats_u += 2 * (size_t)tc_rows_a(J + nbj) * tc_kp(nbj);
    }
    void *pl = nullptr, *pu = nullptr, *pt = nullptr, *pw = nullptr, *ptw = nullptr;
    GRIM_TRY(grim_workspace(h, "gs_l", floats_l * sizeof(float), &pl));
    GRIM_TRY(grim_workspace(h, "gs_u", floats_u * sizeof(float), &pu));
    // diagonal-block inverses live at their own positions of two n x n matrices
    GRIM_TRY(grim_workspace(h, "gs_t", (size_t)2 * n * n * sizeof(float2), &pt));
    GRIM_TRY(grim_workspace(h, "gs_w", (size_t)n * nb * sizeof(float2), &pw));
    GRIM_TRY(grim_workspace(h, "gs_tw", (size_t)n * nb / 2 * sizeof(float2), &ptw));
    float2 *TL = (float2 *)pt, *TU = TL + (size_t)n * n, *W = (float2 *)pw;
    const int64_t ldt = n;
    // full blocks: recursive doubling over all of them at once; a partial last block by
    // 64-row substitution steps
    if (nfull > 0) {
        GRIM_TRY(gs_invert_recursive(h, LU, lda, nfull * nb, nb, TL, ldt, (float2 *)ptw, false));
        GRIM_TRY(gs_invert_recursive(h, LU, lda, nfull * nb, nb, TU, ldt, (float2 *)ptw, true));
    }
    if (nblk > nfull) {
        const int J = nfull * nb, bd = n - J;
        const int64_t off = (int64_t)J * (ldt + 1);
        GRIM_TRY(gs_invert_blocks(h, LU, lda, J, 1, bd, TL + off, ldt, 0, false, nb));
        GRIM_TRY(gs_invert_blocks(h, LU, lda, J, 1, bd, TU + off, ldt, 0, true, nb));
    }
    P->n = n;
    P->nblk = nblk;
    P->nb = nb;
    P->L.assign(nblk, TcPacked{});
    P->U.assign(nblk, TcPacked{});
    float *fl = (float *)pl, *fu = (float *)pu;
    auto pack_rows = [&](const TcPacked &dst, int M, int K, const float2 *A, int64_t ld_a, int r_off, int rows) {
        const int64_t chunks = (int64_t)rows * (dst.kp / 4);
        k_tc_pack_a<<<ceil_div(chunks, 256), 256, 0, h->stream>>>(M, K, A, ld_a, dst.hi, dst.lo, rows, dst.rows_p, r_off,
                                                                  dst.kp, 1.f);
        GRIM_CHECK_LAUNCH_W(h, "k_tc_pack_a", 0.0, 8.0 * M * K + 32.0 * chunks);
        return GRIM_OK;
    };
    for (int i = 0; i < nblk; ++i) {
        const int J = i * nb, nbj = std::min(nb, n - J), kp = tc_kp(nbj);
        const float2 *Ti = TL + (int64_t)J * (ldt + 1), *Ui = TU + (int64_t)J * (ldt + 1);
        // forward panel [Linv; -L_below Linv], rows J..n
        TcPacked &pli = P->L[i];
        pli.hi = fl;
        pli.rows_p = tc_rows_a(n - J);
        pli.kp = kp;
        pli.lo = fl + (size_t)pli.rows_p * kp;
        fl += 2 * (size_t)pli.rows_p * kp;
        const int below = n - J - nbj;
        GRIM_TRY(pack_rows(pli, nbj, nbj, Ti, ldt, 0, below > 0 ? 2 * nbj : pli.rows_p));
        if (below > 0) {
            GRIM_TRY(tc_cgemm(h, below, nbj, nbj, LU + (int64_t)J * lda + J + nbj, lda, Ti, ldt, W, below, -1.f, true));
            GRIM_TRY(pack_rows(pli, below, nbj, W, below, 2 * nbj, pli.rows_p - 2 * nbj));
        }
        // backward panel [-U_above Uinv; Uinv], rows 0..J+nbj
        TcPacked &pui = P->U[i];
        pui.hi = fu;
        pui.rows_p = tc_rows_a(J + nbj);
        pui.kp = kp;
        pui.lo = fu + (size_t)pui.rows_p * kp;
        fu += 2 * (size_t)pui.rows_p * kp;
        if (J > 0) {
            GRIM_TRY(tc_cgemm(h, J, nbj, nbj, LU + (int64_t)J * lda, lda, Ui, ldt, W, J, -1.f, true));
            GRIM_TRY(pack_rows(pui, J, nbj, W, J, 0, 2 * J));
        }
        GRIM_TRY(pack_rows(pui, nbj, nbj, Ui, ldt, 2 * J, pui.rows_p - 2 * J));
    }
    return GRIM_OK;
}

static int gs_apply(grim_context *h, const GsPanels &P, int nrhs, const int *ipiv, const int *ident, float2 *B,
                    int64_t ldb) {
    const int n = P.n, nb = P.nb;
    GRIM_TRY(rhs_interchanges<float2>(h, n, nrhs, B, ldb, ipiv, ident));
    const int bn = h->tune_solve_bn ? h->tune_solve_bn : tc_bn(nrhs), np = ceil_div(nrhs, bn) * bn;
    TcPacked pb;
    GRIM_TRY(tc_ws(h, "gs_b", np, tc_kp(GS_NB_MAX), &pb));
    for (int i = 0; i < P.nblk; ++i) {
        const int J = i * nb, nbj = std::min(nb, n - J);
        pb.kp = P.L[i].kp;
        GRIM_TRY(tc_pack_b(h, nbj, nrhs, B + J, ldb, pb));
        GRIM_TRY(tc_gemm_packed(h, bn, P.L[i], pb, B + J, ldb, n - J, nrhs, nbj, 1.f, 0, nbj));
    }
    for (int i = P.nblk - 1; i >= 0; --i) {
        const int J = i * nb, nbj = std::min(nb, n - J);
        pb.kp = P.U[i].kp;
        GRIM_TRY(tc_pack_b(h, nbj, nrhs, B + J, ldb, pb));
        GRIM_TRY(tc_gemm_packed(h, bn, P.U[i], pb, B, ldb, J + nbj, nrhs, nbj, 1.f, J, J + nbj));
    }
    return GRIM_OK;
}

// The packed-panel solve pays for itself with wide right-hand sides on tensor cores.
static bool gs_wanted(int n, int nrhs) { return tc_enabled() && n >= 512 && nrhs >= 128; }

extern "C" int grim_zgetrf(grim_handle_t h, int n, void *A, int64_t lda, int *ipiv, int *info) {
    return getrf_impl<double2>(h, n, (double2 *)A, lda, ipiv, info);
}
extern "C" int grim_cgetrf(grim_handle_t h, int n, void *A, int64_t lda, int *ipiv, int *info) {
    return getrf_impl<float2>(h, n, (float2 *)A, lda, ipiv, info);
}
extern "C" int grim_zgetrs(grim_handle_t h, int n, int nrhs, const void *LU, int64_t lda, const int *ipiv, void *B,
                           int64_t ldb) {
    return getrs_impl<double2>(h, n, nrhs, (const double2 *)LU, lda, ipiv, (double2 *)B, ldb);
}
extern "C" int grim_cgetrs(grim_handle_t h, int n, int nrhs, const void *LU, int64_t lda, const int *ipiv, void *B,
                           int64_t ldb) {
    return getrs_impl<float2>(h, n, nrhs, (const float2 *)LU, lda, ipiv, (float2 *)B, ldb);
}

// ============================================================== residual / backward error
// R = B - A X (FP64 arithmetic; A complex128 or complex64), then per-column maxima and the
// normwise backward error.  maxes_dev[0] = max berr, [1] = max relative residual.
// Backward error and relative residual per column from an existing residual R.
static int berr_from_residual(grim_context *h, int n, int nrhs, const double2 *R, int64_t ldr, const double2 *X,
                              int64_t ldx, const double2 *B, int64_t ldb, const double *anorm, double *berr,
                              double *relres, double *maxes) {
    void *p = nullptr;
    GRIM_TRY(grim_workspace(h, "berr_absmax", (size_t)3 * nrhs * sizeof(double), &p));
    k_col_absmax3<double2><<<nrhs, 256, 0, h->stream>>>(n, R, ldr, X, ldx, B, ldb, (double *)p);
    GRIM_CHECK_LAUNCH(h, "k_col_absmax3");
    k_berr_finish<<<1, 1024, 0, h->stream>>>(nrhs, (const double *)p, anorm, berr, relres, maxes);
    GRIM_CHECK_LAUNCH(h, "k_berr_finish");
    return GRIM_OK;
}

template <typename TA>
static int residual_and_berr(grim_context *h, int n, int nrhs, const TA *A, int64_t lda, const double2 *X, int64_t ldx,
                             const double2 *B, int64_t ldb, double2 *R, int64_t ldr, const double *anorm, double *berr,
                             double *relres, double *maxes) {
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(R, ldr * sizeof(double2), B, ldb * sizeof(double2), n * sizeof(double2), nrhs,
                                      cudaMemcpyDeviceToDevice, h->stream));
    GRIM_TRY((gemm<double2, TA, double2, double2, true, true>(h, n, nrhs, n, A, lda, X, ldx, R, ldr)));
    return berr_from_residual(h, n, nrhs, R, ldr, X, ldx, B, ldb, anorm, berr, relres, maxes);
}

// ------------------------------------------------ residual on the integer tensor cores
// A~ cut once into S int8 slices (ozaki.cuh); every residual then slices X and runs one
// k_oz_gemm (S accumulators of BN tensor-memory columns).  S = 8 gives an FP64 GEMM's
// accuracy (4e-17 of max |A||X|), S = 7 about 6e-15 with 28 slice pairs instead of 36,
// S = 6 about 1e-12 with 21 pairs (see oz_slices_for).  BN is 64, or 80 for S = 6 when
// that needs fewer waves of CTAs (6 x 80 accumulator columns still fit the 512 of TMEM).
struct OzA {
    int n = 0, S = 0, Rp = 0;
    int8_t *Q = nullptr;
    int *row_exp = nullptr;
};

static inline bool oz_supported(int S) { return S >= 6 && S <= 8; }
// 7 slices leave an error of about 6e-15 of |A||X| in the residual, 6 slices about 1e-12:
// enough for a backward-error target of 1e-13 (7) or 1e-11 (6) and looser, with two
// orders of magnitude to spare.  A relative-residual target (|r| / |b|) is scaled by |b|
// instead, which for an ill-conditioned system is far below |A||X|: 8 slices.
static inline int oz_slices_for(bool berr_test, double tol) {
    if (!berr_test) return 8;
    return tol >= 1e-11 ? 6 : (tol >= 1e-13 ? 7 : 8);
}

// Output-tile width of the slice GEMM: 64, or 80 when S = 6 and the wider tile needs
// fewer waves of CTAs in total time (waves x width, one CTA per SM).
static int oz_bn(int S, int nrhs, int Rp, int sms) {
    if (S != 6) return 64;
    auto cost = [&](int bn) {
        const int64_t tiles = (int64_t)ceil_div(nrhs, bn) * (Rp / 128);
        return (int64_t)ceil_div(tiles, (int64_t)sms) * bn;
    };
    return cost(80) < cost(64) ? 80 : 64;
}

// int32 accumulators hold S products of 2n terms of at most 64^2.
static bool oz_fits(int n, int S) { return (double)S * 2.0 * n * 64.0 * 64.0 < 2147483647.0; }

template <typename TA>
static int oz_prepare_a(grim_context *h, int n, const TA *A, int64_t lda, int S, OzA *out) {
    if (!oz_supported(S)) return grim_fail(GRIM_ERR_ARGUMENT, "integer-slice residual: unsupported slice count");
    const int Rp = ceil_div(2 * n, 128) * 128;
    void *pq = nullptr, *pm = nullptr, *pe = nullptr;
    GRIM_TRY(grim_workspace(h, "oz_q", (size_t)S * Rp * Rp, &pq));
    GRIM_TRY(grim_workspace(h, "oz_rowmax", (size_t)n * sizeof(unsigned long long), &pm));
    GRIM_TRY(grim_workspace(h, "oz_rowexp", (size_t)n * sizeof(int), &pe));
    GRIM_CHECK_CUDA(cudaMemsetAsync(pm, 0, (size_t)n * sizeof(unsigned long long), h->stream));
    k_oz_rowmax<TA><<<dim3(ceil_div(n, 256), 32), 256, 0, h->stream>>>(n, A, lda, (unsigned long long *)pm);
    GRIM_CHECK_LAUNCH(h, "k_oz_rowmax");
    const int64_t threads = (int64_t)(Rp / 2) * (Rp / 16);
    const unsigned long long *rm = (const unsigned long long *)pm;
    if (S == 6)
        k_oz_slice_a<TA, 6><<<ceil_div(threads, 256), 256, 0, h->stream>>>(n, A, lda, rm, (int8_t *)pq, Rp, Rp, (int *)pe);
    else if (S == 7)
        k_oz_slice_a<TA, 7><<<ceil_div(threads, 256), 256, 0, h->stream>>>(n, A, lda, rm, (int8_t *)pq, Rp, Rp, (int *)pe);
    else
        k_oz_slice_a<TA, 8><<<ceil_div(threads, 256), 256, 0, h->stream>>>(n, A, lda, rm, (int8_t *)pq, Rp, Rp, (int *)pe);
    GRIM_CHECK_LAUNCH_W(h, "k_oz_slice_a", 0.0, (double)sizeof(TA) * n * n + (double)S * Rp * Rp);
    out->n = n;
    out->S = S;
    out->Rp = Rp;
    out->Q = (int8_t *)pq;
    out->row_exp = (int *)pe;
    return GRIM_OK;
}

template <int S, int BN>
static int oz_launch(grim_context *h, const OzA &qa, const int8_t *P, int Np, const int *col_exp, const double2 *B,
                     int64_t ldb, double2 *R, int64_t ldr, int nrhs, int *err) {
    using Cfg = OzCfg<S, BN>;
    static PerDeviceOnce attr;
    if (attr.needed()) {
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_oz_gemm<S, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             Cfg::SMEM_BYTES));
        attr.mark();
    }
    dim3 grid(Np / BN, qa.Rp / TC_BM);
    k_oz_gemm<S, BN><<<grid, TC_THREADS, Cfg::SMEM_BYTES, h->stream>>>(
        qa.Rp / OZ_KT, qa.Q, qa.Rp, P, Np, qa.Rp, qa.row_exp, col_exp, (const double *)B, 2 * ldb, (double *)R,
        2 * ldr, 2 * qa.n, nrhs, err);
    GRIM_CHECK_LAUNCH_W(h, "k_oz_gemm", 8.0 * qa.n * qa.n * nrhs,
                        (double)S * qa.Rp * qa.Rp * (Np / BN) + (double)S * Np * qa.Rp * (qa.Rp / TC_BM) +
                            32.0 * qa.n * nrhs);
    return GRIM_OK;
}

// R = B - A X with A prepared by oz_prepare_a (R and B distinct).
static int oz_residual(grim_context *h, const OzA &qa, int nrhs, const double2 *X, int64_t ldx, const double2 *B,
                       int64_t ldb, double2 *R, int64_t ldr) {
    const int n = qa.n, S = qa.S, Kp = qa.Rp;
    const int bn = oz_bn(S, nrhs, qa.Rp, h->sm_count), Np = ceil_div(nrhs, bn) * bn;
    void *pp = nullptr, *pc = nullptr, *pe = nullptr;
    GRIM_TRY(grim_workspace(h, "oz_p", (size_t)S * Np * Kp, &pp));
    GRIM_TRY(grim_workspace(h, "oz_colmax", (size_t)nrhs * sizeof(double), &pc));
    GRIM_TRY(grim_workspace(h, "oz_colexp", (size_t)nrhs * sizeof(int), &pe));
    k_oz_colmax<<<nrhs, 256, 0, h->stream>>>(n, X, ldx, (double *)pc);
    GRIM_CHECK_LAUNCH(h, "k_oz_colmax");
    const int64_t threads = (int64_t)Np * (Kp / 16);
    const double *cm = (const double *)pc;
    int8_t *Pq = (int8_t *)pp;
    int *ce = (int *)pe;
    if (S == 6)
        k_oz_slice_x<6><<<ceil_div(threads, 256), 256, 0, h->stream>>>(n, nrhs, X, ldx, cm, Pq, Np, Kp, ce);
    else if (S == 7)
        k_oz_slice_x<7><<<ceil_div(threads, 256), 256, 0, h->stream>>>(n, nrhs, X, ldx, cm, Pq, Np, Kp, ce);
    else
        k_oz_slice_x<8><<<ceil_div(threads, 256), 256, 0, h->stream>>>(n, nrhs, X, ldx, cm, Pq, Np, Kp, ce);
    GRIM_CHECK_LAUNCH_W(h, "k_oz_slice_x", 0.0, 16.0 * n * nrhs + (double)S * Np * Kp);
    int *err;
    GRIM_TRY(tc_err_flag(h, &err));
    if (S == 6) {
        if (bn == 80) return oz_launch<6, 80>(h, qa, Pq, Np, ce, B, ldb, R, ldr, nrhs, err);
        return oz_launch<6, 64>(h, qa, Pq, Np, ce, B, ldb, R, ldr, nrhs, err);
    }
    if (S == 7) return oz_launch<7, 64>(h, qa, Pq, Np, ce, B, ldb, R, ldr, nrhs, err);
    return oz_launch<8, 64>(h, qa, Pq, Np, ce, B, ldb, R, ldr, nrhs, err);
}

template <typename TA>
static int inf_norm(grim_context *h, int n, const TA *A, int64_t lda, double *anorm_dev) {
    void *p = nullptr, *pp = nullptr;
    GRIM_TRY(grim_workspace(h, "rowsum", (size_t)n * sizeof(double), &p));
    GRIM_TRY(grim_workspace(h, "rowsum_partial", (size_t)n * ROWSUM_CHUNKS * sizeof(double), &pp));
    dim3 g(ceil_div(n, 128), ROWSUM_CHUNKS);
    k_row_abs_partial<TA><<<g, 128, 0, h->stream>>>(n, A, lda, (double *)pp);
    GRIM_CHECK_LAUNCH(h, "k_row_abs_partial");
    k_row_abs_finish<<<ceil_div(n, 128), 128, 0, h->stream>>>(n, (const double *)pp, (double *)p);
    GRIM_CHECK_LAUNCH(h, "k_row_abs_finish");
    k_max_reduce<<<1, 1024, 0, h->stream>>>(n, (const double *)p, anorm_dev);
    GRIM_CHECK_LAUNCH(h, "k_max_reduce");
    return GRIM_OK;
}

extern "C" int grim_backward_error(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, int a_complex64,
                                   const void *X, int64_t ldx, const void *B, int64_t ldb, double *berr_dev) {
    if (!h || n <= 0 || nrhs <= 0 || !A || !X || !B || !berr_dev || lda < n || ldx < n || ldb < n)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_backward_error: bad arguments");
    DeviceGuard g(h->device);
    void *pr = nullptr, *ps = nullptr;
    GRIM_TRY(grim_workspace(h, "be_R", (size_t)n * nrhs * sizeof(double2), &pr));
    GRIM_TRY(grim_workspace(h, "be_scalars", 8 * sizeof(double), &ps));
    double *sc = (double *)ps;
    if (a_complex64) {
        GRIM_TRY(inf_norm(h, n, (const float2 *)A, lda, sc));
        GRIM_TRY(residual_and_berr(h, n, nrhs, (const float2 *)A, lda, (const double2 *)X, ldx, (const double2 *)B, ldb,
                                   (double2 *)pr, n, sc, berr_dev, nullptr, sc + 1));
    } else {
        GRIM_TRY(inf_norm(h, n, (const double2 *)A, lda, sc));
        GRIM_TRY(residual_and_berr(h, n, nrhs, (const double2 *)A, lda, (const double2 *)X, ldx, (const double2 *)B, ldb,
                                   (double2 *)pr, n, sc, berr_dev, nullptr, sc + 1));
    }
    return GRIM_OK;
}

// Test / diagnostic entry: R = B - A X with the FP64 SIMT GEMM (slices 0) or on the integer
// tensor cores with 6, 7 or 8 int8 slices per operand.
extern "C" int grim_residual(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, int a_complex64,
                             const void *X, int64_t ldx, const void *B, int64_t ldb, void *R, int64_t ldr, int slices) {
    if (!h || n <= 0 || nrhs <= 0 || !A || !X || !B || !R || lda < n || ldx < n || ldb < n || ldr < n ||
        (slices != 0 && !oz_supported(slices)) || (slices && !oz_fits(n, slices)))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_residual: bad arguments");
    DeviceGuard g(h->device);
    const double2 *Xd = (const double2 *)X, *Bd = (const double2 *)B;
    double2 *Rd = (double2 *)R;
    if (slices == 0) {
        GRIM_CHECK_CUDA(cudaMemcpy2DAsync(Rd, ldr * sizeof(double2), Bd, ldb * sizeof(double2), n * sizeof(double2),
                                          nrhs, cudaMemcpyDeviceToDevice, h->stream));
        if (a_complex64)
            return gemm<double2, float2, double2, double2, true, true>(h, n, nrhs, n, (const float2 *)A, lda, Xd, ldx,
                                                                       Rd, ldr);
        return gemm<double2, double2, double2, double2, true, true>(h, n, nrhs, n, (const double2 *)A, lda, Xd, ldx, Rd,
                                                                    ldr);
    }
    OzA qa;
    if (a_complex64) GRIM_TRY(oz_prepare_a(h, n, (const float2 *)A, lda, slices, &qa));
    else GRIM_TRY(oz_prepare_a(h, n, (const double2 *)A, lda, slices, &qa));
    GRIM_TRY(oz_residual(h, qa, nrhs, Xd, ldx, Bd, ldb, Rd, ldr));
    return tc_err_check(h, "grim_residual");
}

// Residual and release measures of one modal solution (reference bor/factor.py:289-300,
// ModalFactor.errors): R = B - A X, per-column backward error and 2-norm relative
// residual, their maxima in maxes[0..1].  On the handle's stream, no host synchronisation:
// the int8 tensor-core residual (slices > 0) leaves its error flag to grim_synchronize.
extern "C" int grim_solution_errors(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, const void *X,
                                    int64_t ldx, const void *B, int64_t ldb, void *R, int64_t ldr, int slices,
                                    double *berr_dev, double *relres_dev, double *maxes_dev) {
    if (!h || n <= 0 || nrhs <= 0 || !A || !X || !B || !R || !maxes_dev || lda < n || ldx < n || ldb < n ||
        ldr < n || (slices != 0 && !oz_supported(slices)) || (slices && !oz_fits(n, slices)))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_solution_errors: bad arguments");
    DeviceGuard g(h->device);
    const double2 *Ad = (const double2 *)A, *Xd = (const double2 *)X, *Bd = (const double2 *)B;
    double2 *Rd = (double2 *)R;
    void *ps = nullptr, *pe = nullptr;
    GRIM_TRY(grim_workspace(h, "se_scalars", 8 * sizeof(double), &ps));
    GRIM_TRY(grim_workspace(h, "se_errs5", (size_t)5 * nrhs * sizeof(double), &pe));
    double *anorm = (double *)ps;
    GRIM_TRY(inf_norm(h, n, Ad, lda, anorm));
    if (slices == 0) {
        GRIM_CHECK_CUDA(cudaMemcpy2DAsync(Rd, ldr * sizeof(double2), Bd, ldb * sizeof(double2), n * sizeof(double2),
                                          nrhs, cudaMemcpyDeviceToDevice, h->stream));
        GRIM_TRY((gemm<double2, double2, double2, double2, true, true>(h, n, nrhs, n, Ad, lda, Xd, ldx, Rd, ldr)));
    } else {
        OzA qa;
        GRIM_TRY(oz_prepare_a(h, n, Ad, lda, slices, &qa));
        GRIM_TRY(oz_residual(h, qa, nrhs, Xd, ldx, Bd, ldb, Rd, ldr));
    }
    k_col_errs5<<<nrhs, 256, 0, h->stream>>>(n, Rd, ldr, Xd, ldx, Bd, ldb, (double *)pe);
    GRIM_CHECK_LAUNCH(h, "k_col_errs5");
    k_errs_finish<<<1, 1024, 0, h->stream>>>(nrhs, (const double *)pe, anorm, berr_dev, relres_dev, maxes_dev);
    GRIM_CHECK_LAUNCH(h, "k_errs_finish");
    return GRIM_OK;
}

// ============================================================== solve (FP64 or mixed)
template <typename TA>
static int mixed_refine(grim_context *h, int n, int nrhs, const TA *Ares, int64_t ldres, float2 *lu32, const int *ipiv,
                        double2 *Bio, int64_t ldb, double tol, int max_iter, grim_solve_info *st,
                        bool berr_test = false) {
    // Bio holds B on entry and X on exit.
    void *pB = nullptr, *pX = nullptr, *pR = nullptr, *pR32 = nullptr, *pS = nullptr;
    GRIM_TRY(grim_workspace(h, "mx_B", (size_t)n * nrhs * sizeof(double2), &pB));
    GRIM_TRY(grim_workspace(h, "mx_X", (size_t)n * nrhs * sizeof(double2), &pX));
    GRIM_TRY(grim_workspace(h, "mx_R", (size_t)n * nrhs * sizeof(double2), &pR));
    GRIM_TRY(grim_workspace(h, "mx_R32", (size_t)n * nrhs * sizeof(float2), &pR32));
    GRIM_TRY(grim_workspace(h, "mx_scalars", 16 * sizeof(double), &pS));
    double2 *B0 = (double2 *)pB, *X = (double2 *)pX, *R = (double2 *)pR;
    float2 *R32 = (float2 *)pR32;
    double *sc = (double *)pS;  // [0] anorm, [1] max berr, [2] max relres
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(B0, n * sizeof(double2), Bio, ldb * sizeof(double2), n * sizeof(double2), nrhs,
                                      cudaMemcpyDeviceToDevice, h->stream));
    GRIM_TRY(inf_norm(h, n, Ares, ldres, sc));
    dim3 eg(ceil_div(n, 256), nrhs);
    // x0 = solve32(b); the diagonal-block inverses are formed once for every solve
    int *ident;
    GRIM_TRY(smem_opt_in<float2>());
    GRIM_TRY(getrs_prepare<float2>(h, n, ipiv, &ident));
    GsPanels panels;
    // the packed-panel solve multiplies by explicitly inverted 512-row triangular blocks: fast,
    // and accurate for diagonally dominant factors; partial-pivoting factors (the
    // combined-field systems) keep the substitution solve, whose first backward error is
    // two orders of magnitude smaller there (one refinement step saved)
    // the explicit block inverses start the refinement at a larger backward error than
    // substitution (2e-3 against 3e-5 at N=2048 on the combined-field systems) and still
    // finish first: one more refinement step costs less than the substitution chain
    const bool use_gs = gs_wanted(n, nrhs);
    if (use_gs) GRIM_TRY(gs_build(h, n, lu32, n, h->tune_gs_block ? h->tune_gs_block : gs_block(n, nrhs), &panels));
    auto solve32 = [&](float2 *X32) -> int {
        if (use_gs) return gs_apply(h, panels, nrhs, ipiv, ident, X32, n);
        return getrs_apply<float2>(h, n, nrhs, lu32, n, ipiv, ident, X32, n);
    };
    k_convert<float2, double2><<<eg, 256, 0, h->stream>>>(n, nrhs, B0, n, R32, n);
    GRIM_CHECK_LAUNCH(h, "k_convert");
    GRIM_TRY(solve32(R32));
    k_convert<double2, float2><<<eg, 256, 0, h->stream>>>(n, nrhs, R32, n, X, n);
    GRIM_CHECK_LAUNCH(h, "k_convert");
    double prev = INFINITY;
    int steps = 0;
    double berr = INFINITY, relres = INFINITY, first = -1.0;
    int status = GRIM_OK;
    // residuals on the integer tensor cores when the slice accumulators fit
    OzA qa;
    const int oz_s = oz_slices_for(berr_test, tol);
    const bool use_oz = tc_enabled() && n >= 256 && nrhs >= 16 && oz_fits(n, oz_s);
    if (use_oz) GRIM_TRY(oz_prepare_a(h, n, Ares, ldres, oz_s, &qa));
    // A backward-error target below complex64 accuracy always needs a correction: the first
    // one is then queued without reading the initial residual's norms on the host (they
    // are kept on the device and read together with the next ones), which saves one host
    // round trip per solve.
    const bool speculate = berr_test && tol < 1e-8 && max_iter > 0;
    for (int it = 0; it <= max_iter; ++it) {
        if (use_oz) {
            GRIM_TRY(oz_residual(h, qa, nrhs, X, n, B0, n, R, n));
            GRIM_TRY(berr_from_residual(h, n, nrhs, R, n, X, n, B0, n, sc, nullptr, nullptr, sc + 1));
        } else {
            GRIM_TRY(residual_and_berr(h, n, nrhs, Ares, ldres, X, n, B0, n, R, n, sc, nullptr, nullptr, sc + 1));
        }
        if (speculate && it == 0) {
            GRIM_CHECK_CUDA(cudaMemcpyAsync(sc + 4, sc + 1, 2 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            k_convert<float2, double2><<<eg, 256, 0, h->stream>>>(n, nrhs, R, n, R32, n);
            GRIM_CHECK_LAUNCH(h, "k_convert");
            GRIM_TRY(solve32(R32));
            k_add_update<float2><<<eg, 256, 0, h->stream>>>(n, nrhs, X, n, R32, n);
            GRIM_CHECK_LAUNCH(h, "k_add_update");
            ++steps;
            continue;
        }
        double hv[4];
        GRIM_CHECK_CUDA(cudaMemcpyAsync(hv, sc + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        if (speculate && it == 1)
            GRIM_CHECK_CUDA(cudaMemcpyAsync(hv + 2, sc + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
        GRIM_TRY(tc_err_check(h, "mixed-precision solve"));
        berr = hv[0];
        relres = hv[1];
        if (speculate && it == 1) {
            first = hv[2];
            prev = berr_test ? hv[2] : hv[3];
            if (!std::isfinite(prev)) {
                status = grim_fail(GRIM_ERR_NOT_CONVERGED, "mixed-precision refinement stalled; double LU required");
                break;
            }
        }
        if (first < 0) first = berr;
        const double measure = berr_test ? berr : relres;
        if (std::isfinite(measure) && measure <= tol) break;
        if (!std::isfinite(measure) || measure >= prev * 0.98) {
            status = grim_fail(GRIM_ERR_NOT_CONVERGED, "mixed-precision refinement stalled; double LU required");
            break;
        }
        if (it == max_iter) {
            status = grim_fail(GRIM_ERR_NOT_CONVERGED, "mixed-precision refinement exceeded its correction limit");
            break;
        }
        prev = measure;
        k_convert<float2, double2><<<eg, 256, 0, h->stream>>>(n, nrhs, R, n, R32, n);
        GRIM_CHECK_LAUNCH(h, "k_convert");
        GRIM_TRY(solve32(R32));
        k_add_update<float2><<<eg, 256, 0, h->stream>>>(n, nrhs, X, n, R32, n);
        GRIM_CHECK_LAUNCH(h, "k_add_update");
        ++steps;
    }
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(Bio, ldb * sizeof(double2), X, n * sizeof(double2), n * sizeof(double2), nrhs,
                                      cudaMemcpyDeviceToDevice, h->stream));
    st->backward_error = berr;
    st->initial_backward_error = first;
    st->refinement_steps = steps;
    return status;
}

extern "C" int grim_zgesv_mixed(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, const void *A32,
                                int64_t lda32, void *B, int64_t ldb, int precision_mode, double tol, int max_iter,
                                int *info, grim_solve_info *stats) {
    const int pivot_req = (precision_mode & GRIM_PREC_TOURNAMENT_PIVOT) ? GRIM_PIVOT_TOURNAMENT
                          : (precision_mode & GRIM_PREC_PARTIAL_PIVOT)  ? GRIM_PIVOT_PARTIAL
                          : (precision_mode & GRIM_PREC_STATIC_PIVOT)   ? GRIM_PIVOT_STATIC
                                                                        : -1;
    precision_mode &= ~(GRIM_PREC_STATIC_PIVOT | GRIM_PREC_PARTIAL_PIVOT | GRIM_PREC_TOURNAMENT_PIVOT);
    if (!h || n <= 0 || nrhs <= 0 || !B || ldb < n || (!A && !A32) || (A && lda < n) || (A32 && lda32 < n) ||
        (precision_mode != GRIM_PREC_FP64 && precision_mode != GRIM_PREC_MIXED &&
         precision_mode != GRIM_PREC_MIXED_BERR))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_zgesv_mixed: bad arguments");
    struct PivotScope {  // a pivot bit applies to this call's factorization only
        grim_context *h;
        int keep;
        PivotScope(grim_context *hh, int mode) : h(hh), keep(hh->pivot_mode) { if (mode >= 0) h->pivot_mode = mode; }
        ~PivotScope() { h->pivot_mode = keep; }
    } scope(h, pivot_req);
    if (precision_mode == GRIM_PREC_FP64 && !A)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_zgesv_mixed: FP64 mode needs the complex128 matrix");
    DeviceGuard g(h->device);
    grim_solve_info st{};
    st.precision_mode = precision_mode;
    int linfo = 0;
    void *pipiv = nullptr;
    GRIM_TRY(grim_workspace(h, "sv_ipiv", (size_t)n * sizeof(int), &pipiv));
    int *ipiv = (int *)pipiv;
    if (precision_mode == GRIM_PREC_FP64) {
        void *plu = nullptr;
        GRIM_TRY(grim_workspace(h, "sv_lu64", (size_t)n * n * sizeof(double2), &plu));
        double2 *lu = (double2 *)plu;
        GRIM_CHECK_CUDA(cudaMemcpy2DAsync(lu, n * sizeof(double2), A, lda * sizeof(double2), n * sizeof(double2), n,
                                          cudaMemcpyDeviceToDevice, h->stream));
        StreamTimer tf(h->stream);
        GRIM_TRY(getrf_impl<double2>(h, n, lu, n, ipiv, &linfo));
        st.ms_factor = tf.stop_ms();
        st.pivoted_panels = h->last.pivoted_panels;
        if (linfo > 0) {
            st.info = linfo;
            h->last = st;
            if (info) *info = linfo;
            return grim_fail(GRIM_ERR_SINGULAR, "grim_zgesv_mixed: matrix is exactly singular");
        }
        StreamTimer ts(h->stream);
        GRIM_TRY(getrs_impl<double2>(h, n, nrhs, lu, n, ipiv, (double2 *)B, ldb));
        st.ms_solve = ts.stop_ms();
        st.backward_error = -1.0;
    } else {
        void *plu = nullptr;
        GRIM_TRY(grim_workspace(h, "sv_lu32", (size_t)n * n * sizeof(float2), &plu));
        float2 *lu = (float2 *)plu;
        if (A32) {
            GRIM_CHECK_CUDA(cudaMemcpy2DAsync(lu, n * sizeof(float2), A32, lda32 * sizeof(float2), n * sizeof(float2), n,
                                              cudaMemcpyDeviceToDevice, h->stream));
        } else {
            dim3 eg(ceil_div(n, 256), n);
            k_convert<float2, double2><<<eg, 256, 0, h->stream>>>(n, n, (const double2 *)A, lda, lu, n);
            GRIM_CHECK_LAUNCH(h, "k_convert");
        }
        // the factorization's flags are read after the refinement's first host synchronisation,
        // so that the solves are queued while the factorization still runs
        StreamTimer tf(h->stream);
        GRIM_TRY(getrf_impl<float2>(h, n, lu, n, ipiv, &linfo, true));
        tf.record();
        StreamTimer ts(h->stream);
        int s;
        const bool berr_test = precision_mode == GRIM_PREC_MIXED_BERR;
        if (A)
            s = mixed_refine<double2>(h, n, nrhs, (const double2 *)A, lda, lu, ipiv, (double2 *)B, ldb, tol, max_iter, &st,
                                      berr_test);
        else
            s = mixed_refine<float2>(h, n, nrhs, (const float2 *)A32, lda32, lu, ipiv, (double2 *)B, ldb, tol, max_iter,
                                     &st, berr_test);
        st.ms_solve = ts.stop_ms();
        st.ms_factor = tf.elapsed_ms();
        int piv = 0;
        GRIM_TRY(getrf_read_flags(h, &linfo, &piv));
        st.pivoted_panels = piv;
        if (linfo > 0) {
            st.info = linfo;
            h->last = st;
            if (info) *info = linfo;
            return grim_fail(GRIM_ERR_SINGULAR, "grim_zgesv_mixed: complex64 factor is exactly singular");
        }
        h->last = st;
        if (stats) *stats = st;
        if (info) *info = 0;
        return s;
    }
    h->last = st;
    if (stats) *stats = st;
    if (info) *info = linfo;
    return GRIM_OK;
}

// FP64 solve of the RCS path with the reference's dense gate: LU in the requested pivot
// mode, the solution's per-column normwise backward error |r| / (|A| |x| + |b|), at most
// max_refine FP64 refinement steps with the same factors while the largest exceeds tol
// (each kept only if it lowers it), and, when the gate still fails or the factors are not
// finite, a certified factorization (LAPACK getrf's pivots) and solve.
extern "C" int grim_zgesv_guarded(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, void *B, int64_t ldb,
                                  int pivot, double tol, int max_refine, double *berr_dev, int *info,
                                  grim_solve_info *stats) {
    if (!h || n <= 0 || nrhs <= 0 || !A || lda < n || !B || ldb < n || !(tol > 0) || max_refine < 0 ||
        pivot < GRIM_PIVOT_CERTIFIED || pivot > GRIM_PIVOT_TOURNAMENT)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_zgesv_guarded: bad arguments");
    DeviceGuard g(h->device);
    grim_solve_info st{};
    st.precision_mode = GRIM_PREC_FP64;
    void *pipiv = nullptr, *plu = nullptr, *pB0 = nullptr, *pR = nullptr, *pS = nullptr, *pbe = nullptr;
    GRIM_TRY(grim_workspace(h, "sv_ipiv", (size_t)n * sizeof(int), &pipiv));
    GRIM_TRY(grim_workspace(h, "sv_lu64", (size_t)n * n * sizeof(double2), &plu));
    GRIM_TRY(grim_workspace(h, "gd_B0", (size_t)n * nrhs * sizeof(double2), &pB0));
    GRIM_TRY(grim_workspace(h, "gd_R", (size_t)n * nrhs * sizeof(double2), &pR));
    GRIM_TRY(grim_workspace(h, "gd_scalars", 8 * sizeof(double), &pS));
    if (!berr_dev) {
        GRIM_TRY(grim_workspace(h, "gd_berr", (size_t)nrhs * sizeof(double), &pbe));
        berr_dev = (double *)pbe;
    }
    int *ipiv = (int *)pipiv;
    double2 *lu = (double2 *)plu, *B0 = (double2 *)pB0, *R = (double2 *)pR, *X = (double2 *)B;
    double *sc = (double *)pS;  // [0] |A|_inf, [1] max berr, [2] max relres
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(B0, n * sizeof(double2), B, ldb * sizeof(double2), n * sizeof(double2), nrhs,
                                      cudaMemcpyDeviceToDevice, h->stream));
    GRIM_TRY(inf_norm(h, n, (const double2 *)A, lda, sc));
    dim3 eg(ceil_div(n, 256), nrhs);
    const int keep = h->pivot_mode;
    double berr = INFINITY;
    int status = GRIM_OK;
    for (int attempt = 0; attempt < 2 && status == GRIM_OK; ++attempt) {
        // attempt 0: the requested pivots; attempt 1: certified (LAPACK getrf's pivots)
        h->pivot_mode = attempt == 0 ? pivot : GRIM_PIVOT_CERTIFIED;
        int linfo = 0;
        GRIM_CHECK_CUDA(cudaMemcpy2DAsync(lu, n * sizeof(double2), A, lda * sizeof(double2), n * sizeof(double2), n,
                                          cudaMemcpyDeviceToDevice, h->stream));
        StreamTimer tf(h->stream);
        status = getrf_impl<double2>(h, n, lu, n, ipiv, &linfo);
        h->pivot_mode = keep;
        if (status != GRIM_OK) break;
        st.ms_factor += tf.stop_ms();
        // after a fallback, -1 - (panels that pivoted) records it
        st.pivoted_panels = attempt == 0 ? h->last.pivoted_panels : -1 - h->last.pivoted_panels;
        if (linfo > 0) {
            if (attempt == 0) continue;  // an exact zero pivot: the pivoted factorization decides
            st.info = linfo;
            h->last = st;
            if (info) *info = linfo;
            return grim_fail(GRIM_ERR_SINGULAR, "grim_zgesv_guarded: matrix is exactly singular");
        }
        StreamTimer ts(h->stream);
        if (attempt == 1)
            GRIM_CHECK_CUDA(cudaMemcpy2DAsync(X, ldb * sizeof(double2), B0, n * sizeof(double2), n * sizeof(double2),
                                              nrhs, cudaMemcpyDeviceToDevice, h->stream));
        GRIM_TRY(getrs_impl<double2>(h, n, nrhs, lu, n, ipiv, X, ldb));
        GRIM_TRY(residual_and_berr(h, n, nrhs, (const double2 *)A, lda, X, ldb, B0, n, R, n, sc, berr_dev, nullptr,
                                   sc + 1));
        double hv = INFINITY;
        GRIM_CHECK_CUDA(cudaMemcpyAsync(&hv, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
        berr = hv;
        if (attempt == 0) st.initial_backward_error = berr;
        for (int it = 0; it < max_refine && std::isfinite(berr) && berr > tol; ++it) {
            // candidate x + solve(r): kept only if it lowers the largest backward error
            void *pc = nullptr, *pcb = nullptr;
            GRIM_TRY(grim_workspace(h, "gd_cand", (size_t)n * nrhs * sizeof(double2), &pc));
            GRIM_TRY(grim_workspace(h, "gd_cand_berr", (size_t)nrhs * sizeof(double), &pcb));
            double2 *Xc = (double2 *)pc;
            GRIM_TRY(getrs_impl<double2>(h, n, nrhs, lu, n, ipiv, R, n));
            GRIM_CHECK_CUDA(cudaMemcpy2DAsync(Xc, n * sizeof(double2), X, ldb * sizeof(double2), n * sizeof(double2),
                                              nrhs, cudaMemcpyDeviceToDevice, h->stream));
            k_add_update<double2><<<eg, 256, 0, h->stream>>>(n, nrhs, Xc, n, R, n);
            GRIM_CHECK_LAUNCH(h, "k_add_update");
            GRIM_TRY(residual_and_berr(h, n, nrhs, (const double2 *)A, lda, Xc, n, B0, n, R, n, sc,
                                       (double *)pcb, nullptr, sc + 2));
            GRIM_CHECK_CUDA(cudaMemcpyAsync(&hv, sc + 2, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
            if (!(hv < berr)) break;
            berr = hv;
            GRIM_CHECK_CUDA(cudaMemcpy2DAsync(X, ldb * sizeof(double2), Xc, n * sizeof(double2), n * sizeof(double2),
                                              nrhs, cudaMemcpyDeviceToDevice, h->stream));
            GRIM_CHECK_CUDA(cudaMemcpyAsync(berr_dev, pcb, nrhs * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            st.refinement_steps += 1;
        }
        st.ms_solve += ts.stop_ms();
        if (std::isfinite(berr) && berr <= tol) break;
    }
    h->pivot_mode = keep;
    GRIM_TRY(status);
    st.backward_error = berr;
    h->last = st;
    if (stats) *stats = st;
    if (info) *info = 0;
    if (!std::isfinite(berr)) return grim_fail(GRIM_ERR_NONFINITE, "grim_zgesv_guarded: non-finite backward error");
    return GRIM_OK;
}

// Mixed-precision solve that reuses an existing complex64 factorization (LU32, ipiv from
// grim_cgetrf with leading dimension n): FP64 refinement against A (complex128) or the
// exact promotion of A32.  Used by the serving engine's resident factor cache.
extern "C" int grim_zgesv_mixed_factored(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda,
                                         const void *A32, int64_t lda32, void *LU32, const int *ipiv, void *B,
                                         int64_t ldb, double tol, int max_iter, grim_solve_info *stats) {
    if (!h || n <= 0 || nrhs <= 0 || !B || ldb < n || (!A && !A32) || (A && lda < n) || (A32 && lda32 < n) || !LU32 ||
        !ipiv)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_zgesv_mixed_factored: bad arguments");
    DeviceGuard g(h->device);
    grim_solve_info st{};
    st.precision_mode = GRIM_PREC_MIXED;
    StreamTimer ts(h->stream);
    int s;
    if (A)
        s = mixed_refine<double2>(h, n, nrhs, (const double2 *)A, lda, (float2 *)LU32, ipiv, (double2 *)B, ldb, tol,
                                  max_iter, &st);
    else
        s = mixed_refine<float2>(h, n, nrhs, (const float2 *)A32, lda32, (float2 *)LU32, ipiv, (double2 *)B, ldb, tol,
                                 max_iter, &st);
    st.ms_solve = ts.stop_ms();
    h->last = st;
    if (stats) *stats = st;
    return s;
}

// ============================================================== condition estimate
// cond_1 of the row/column-equilibrated matrix (the reference's condition_est; kernels and
// the estimator's description in condest.cuh).  B^-1 v = C A^-1 R v and B^-H v = R A^-H C v
// run on partial-pivoting LUs of A and of A^H; the iteration is LAPACK zlacn2's.
extern "C" int grim_zcond1_equilibrated(grim_handle_t h, int n, const void *A, int64_t lda, double *cond) {
    if (!h || n <= 0 || !A || lda < n || !cond) return grim_fail(GRIM_ERR_ARGUMENT, "grim_zcond1_equilibrated: bad arguments");
    DeviceGuard g(h->device);
    struct PivotScope {
        grim_context *h;
        int keep;
        explicit PivotScope(grim_context *hh) : h(hh), keep(hh->pivot_mode) { h->pivot_mode = GRIM_PIVOT_PARTIAL; }
        ~PivotScope() { h->pivot_mode = keep; }
    } scope(h);
    void *plu = nullptr, *pluh = nullptr, *pip = nullptr, *pr = nullptr, *pc = nullptr, *pv = nullptr, *ps = nullptr;
    GRIM_TRY(grim_workspace(h, "cond_lu", (size_t)n * n * sizeof(double2), &plu));
    GRIM_TRY(grim_workspace(h, "cond_luh", (size_t)n * n * sizeof(double2), &pluh));
    GRIM_TRY(grim_workspace(h, "cond_ipiv", (size_t)2 * n * sizeof(int), &pip));
    GRIM_TRY(grim_workspace(h, "cond_rmax", (size_t)n * sizeof(unsigned long long), &pr));
    GRIM_TRY(grim_workspace(h, "cond_cols", (size_t)2 * n * sizeof(double), &pc));
    GRIM_TRY(grim_workspace(h, "cond_vec", (size_t)2 * n * sizeof(double2), &pv));
    GRIM_TRY(grim_workspace(h, "cond_scal", 64, &ps));
    double2 *lu = (double2 *)plu, *luh = (double2 *)pluh, *x = (double2 *)pv;
    int *ipiv = (int *)pip, *ipivh = ipiv + n;
    unsigned long long *rmax = (unsigned long long *)pr;
    double *cscale = (double *)pc, *colsum = cscale + n;
    double *sd = (double *)ps;
    int *si = (int *)(sd + 4);
    const double2 *a = (const double2 *)A;

    // equilibration and ||B||_1
    GRIM_CHECK_CUDA(cudaMemsetAsync(rmax, 0, (size_t)n * sizeof(unsigned long long), h->stream));
    const int chunk = 64;
    k_cond_rowmax<<<dim3(ceil_div(n, 256), ceil_div(n, chunk)), 256, 0, h->stream>>>(n, a, lda, chunk, rmax);
    GRIM_CHECK_LAUNCH(h, "k_cond_rowmax");
    k_cond_cols<<<n, 256, 0, h->stream>>>(n, a, lda, rmax, cscale, colsum);
    GRIM_CHECK_LAUNCH(h, "k_cond_cols");
    k_cond_max<<<1, 1024, 0, h->stream>>>(n, colsum, sd);
    GRIM_CHECK_LAUNCH(h, "k_cond_max");

    // LUs of A and A^H
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(lu, n * sizeof(double2), a, lda * sizeof(double2), n * sizeof(double2), n,
                                      cudaMemcpyDeviceToDevice, h->stream));
    int info = 0, infoh = 0;
    GRIM_TRY(getrf_impl<double2>(h, n, lu, n, ipiv, &info));
    k_conj_transpose<<<dim3(ceil_div(n, 32), ceil_div(n, 32)), dim3(32, 8), 0, h->stream>>>(n, a, lda, luh, n);
    GRIM_CHECK_LAUNCH(h, "k_conj_transpose");
    GRIM_TRY(getrf_impl<double2>(h, n, luh, n, ipivh, &infoh));
    double norm_b = 0.0;
    GRIM_CHECK_CUDA(cudaMemcpyAsync(&norm_b, sd, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (info > 0 || infoh > 0 || !std::isfinite(norm_b)) {
        *cond = INFINITY;  // exactly singular (or non-finite entries)
        return GRIM_OK;
    }

    const int vb = ceil_div(n, 256);
    auto binv = [&](bool adjoint) -> int {  // x <- B^-1 x or B^-H x
        k_cond_scale<<<vb, 256, 0, h->stream>>>(n, x, adjoint ? cscale : nullptr, adjoint ? nullptr : rmax);
        GRIM_CHECK_LAUNCH(h, "k_cond_scale");
        GRIM_TRY(getrs_impl<double2>(h, n, 1, adjoint ? luh : lu, n, adjoint ? ipivh : ipiv, x, n));
        k_cond_scale<<<vb, 256, 0, h->stream>>>(n, x, adjoint ? nullptr : cscale, adjoint ? rmax : nullptr);
        GRIM_CHECK_LAUNCH(h, "k_cond_scale");
        return GRIM_OK;
    };
    auto fill = [&](int mode, int j) {
        k_cond_fill<<<vb, 256, 0, h->stream>>>(n, x, mode, j);
        return grim_launch_status(h, "k_cond_fill", 0, 0);
    };
    auto norm_sign = [&](bool sign, double *out) -> int {  // ||x||_1 (x <- sign(x) when asked)
        k_cond_norm_sign<<<1, 1024, 0, h->stream>>>(n, x, sign ? x : nullptr, sd + 1);
        GRIM_CHECK_LAUNCH(h, "k_cond_norm_sign");
        GRIM_CHECK_CUDA(cudaMemcpyAsync(out, sd + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
        return GRIM_OK;
    };
    auto argmax = [&](int jlast, int *j, double *zj, double *zlast) -> int {
        k_cond_argmax<<<1, 1024, 0, h->stream>>>(n, x, jlast, si, sd + 2);
        GRIM_CHECK_LAUNCH(h, "k_cond_argmax");
        double d[2];
        GRIM_CHECK_CUDA(cudaMemcpyAsync(j, si, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        GRIM_CHECK_CUDA(cudaMemcpyAsync(d, sd + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
        *zj = d[0];
        *zlast = d[1];
        return GRIM_OK;
    };

    // zlacn2: x = (1/n) e; y = B^-1 x
    double est = 0.0;
    GRIM_TRY(fill(0, 0));
    GRIM_TRY(binv(false));
    if (n == 1) {
        GRIM_TRY(norm_sign(false, &est));
    } else {
        GRIM_TRY(norm_sign(true, &est));  // x = sign(y)
        GRIM_TRY(binv(true));              // z = B^-H x
        int j = 0, iter = 2;
        double zj = 0.0, zl = 0.0;
        GRIM_TRY(argmax(-1, &j, &zj, &zl));
        for (;;) {
            GRIM_TRY(fill(1, j));  // x = e_j
            GRIM_TRY(binv(false));
            const double old = est;
            GRIM_TRY(norm_sign(true, &est));
            if (!(est > old)) {
                est = std::max(est, old);
                break;
            }
            GRIM_TRY(binv(true));
            const int jlast = j;
            GRIM_TRY(argmax(jlast, &j, &zj, &zl));
            if (zl != zj && iter < 5) {
                ++iter;
                continue;
            }
            break;
        }
        // the alternating-sign test vector
        GRIM_TRY(fill(2, 0));
        GRIM_TRY(binv(false));
        double alt = 0.0;
        GRIM_TRY(norm_sign(false, &alt));
        alt = 2.0 * alt / (3.0 * n);
        if (alt > est) est = alt;
    }
    const double c = norm_b * est;
    *cond = std::isfinite(c) ? c : INFINITY;
    return GRIM_OK;
}

// ------------------------------------------------ condition estimates of factored systems
extern "C" int grim_zcond1_factored(grim_handle_t h, int count, const grim_cond_system *sys, double *cond_dev) {
    if (!h || count <= 0 || count > 65535 || !sys || !cond_dev)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_zcond1_factored: bad arguments");
    DeviceGuard g(h->device);
    std::vector<CondSysDev> d(count);
    size_t tot = 0;
    int nmax = 0;
    for (int i = 0; i < count; ++i) {
        const grim_cond_system &q = sys[i];
        bool ok = q.n > 0 && q.A && q.lda >= q.n && q.lu[0];
        if (ok && q.halves) {
            const int ke = q.k + q.nfe, ko = q.k + q.nfo;
            ok = q.k >= 0 && q.nfe >= 0 && q.nfo >= 0 && ke > 0 && ko > 0 && 2 * q.k + q.nfe + q.nfo == q.n &&
                 q.lu[1] && q.ipiv[0] && q.ipiv[1] && q.ldlu[0] >= ke && q.ldlu[1] >= ko &&
                 (q.k == 0 || (q.p1 && q.p2 && q.s)) && (q.nfe == 0 || q.fe) && (q.nfo == 0 || q.fo);
        } else if (ok) {
            ok = q.ldlu[0] >= q.n;
        }
        if (!ok) return grim_fail(GRIM_ERR_ARGUMENT, "grim_zcond1_factored: bad system description");
        tot += (size_t)q.n;
        nmax = std::max(nmax, q.n);
    }
    void *ps = nullptr, *pv = nullptr, *pc = nullptr;
    GRIM_TRY(grim_workspace(h, "mc_sys", (size_t)count * sizeof(CondSysDev), &ps));
    GRIM_TRY(grim_workspace(h, "mc_vec", 2 * tot * sizeof(double2), &pv));
    GRIM_TRY(grim_workspace(h, "mc_colsum", tot * sizeof(double), &pc));
    double2 *vec = (double2 *)pv;
    double *colsum = (double *)pc;
    size_t off = 0;
    for (int i = 0; i < count; ++i) {
        const grim_cond_system &q = sys[i];
        CondSysDev &e = d[i];
        e.n = q.n;
        e.halves = q.halves ? 1 : 0;
        e.lu_c64[0] = q.lu_complex64 & 1;
        e.lu_c64[1] = q.halves ? (q.lu_complex64 >> 1) & 1 : 0;
        e.order[0] = q.halves ? q.k + q.nfe : q.n;
        e.order[1] = q.halves ? q.k + q.nfo : 0;
        e.lu[0] = q.lu[0];
        e.lu[1] = q.halves ? q.lu[1] : nullptr;
        e.ld[0] = q.ldlu[0];
        e.ld[1] = q.halves ? q.ldlu[1] : 0;
        e.ipiv[0] = q.halves ? q.ipiv[0] : nullptr;
        e.ipiv[1] = q.halves ? q.ipiv[1] : nullptr;
        e.k = q.halves ? q.k : 0;
        e.nfe = q.halves ? q.nfe : 0;
        e.nfo = q.halves ? q.nfo : 0;
        e.p1 = q.p1;
        e.p2 = q.p2;
        e.fe = q.fe;
        e.fo = q.fo;
        e.s = q.s;
        e.a = (const double2 *)q.A;
        e.lda = q.lda;
        e.colsum = colsum + off;
        e.x = vec + 2 * off;
        e.w = vec + 2 * off + q.n;
        off += (size_t)q.n;
    }
    CondSysDev *dsys = (CondSysDev *)ps;
    GRIM_CHECK_CUDA(cudaMemcpyAsync(dsys, d.data(), (size_t)count * sizeof(CondSysDev), cudaMemcpyHostToDevice,
                                    h->stream));
    k_cond_colsum<<<dim3(ceil_div(nmax, 8), count), 256, 0, h->stream>>>(dsys);
    GRIM_CHECK_LAUNCH(h, "k_cond_colsum");
    k_cond_lacn2<<<count, CS_THREADS, 0, h->stream>>>(dsys, cond_dev);
    GRIM_CHECK_LAUNCH(h, "k_cond_lacn2");
    return GRIM_OK;
}

// ============================================================== grouped factorization
// Schedule of one grouped factorization (grouped.cuh): systems sorted by decreasing order;
// per 64-column step p the number of active systems, of systems with a trailing matrix,
// and, for the latter, prefix sums of the CTA counts of the panel solve, the operand
// packing and the trailing update (offsets into one int array).
struct GrpPlan {
    std::vector<int> order;                 // sorted position -> caller's index
    std::vector<int> active, upd;           // per step
    std::vector<int> off, tot;              // 3 per step: apply, pack, update
    std::vector<double> fl_diag, fl_apply, fl_upd;
    std::vector<int> sched;
    int nmax = 0;
    int bn = 128;  // output-tile width of the complex64 trailing update
};

// Output-tile width of the grouped complex64 trailing update (C staged in shared memory in
// both): 128 (two pipeline stages, one CTA per SM) or 64 (one stage, 81 KB, two CTAs per SM so
// that one CTA's loads and epilogue overlap the other's).  GRIM_GROUPED_BN selects it; the
// packed operands are padded for either.
static int grp_bn() {
    static int bn = [] {
        const char *e = getenv("GRIM_GROUPED_BN");
        return (e && atoi(e) == 64) ? 64 : 128;
    }();
    return bn;
}

// The complex64 trailing update runs as the persistent kernel (one CTA per SM walking the
// step's tiles) unless GRIM_GROUPED_PERSIST=0 (one CTA per tile).
static bool grp_persistent() {
    static bool on = [] {
        const char *e = getenv("GRIM_GROUPED_PERSIST");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

template <typename C>
static int grp_plan(int count, const int *n, int bn, GrpPlan *P) {
    P->bn = bn;
    P->order.resize(count);
    for (int i = 0; i < count; ++i) P->order[i] = i;
    std::stable_sort(P->order.begin(), P->order.end(), [&](int a, int b) { return n[a] > n[b]; });
    P->nmax = n[P->order[0]];
    const int steps = ceil_div(P->nmax, NB);
    P->active.assign(steps, 0);
    for (int i = 0; i < count; ++i)
        for (int p = 0; p < ceil_div(n[i], NB); ++p) P->active[p]++;
    P->upd.assign(steps, 0);
    for (int p = 0; p + 1 < steps; ++p) P->upd[p] = P->active[p + 1];
    P->off.assign(3 * steps, 0);
    P->tot.assign(3 * steps, 0);
    P->fl_diag.assign(steps, 0.0);
    P->fl_apply.assign(steps, 0.0);
    P->fl_upd.assign(steps, 0.0);
    P->sched.clear();
    for (int p = 0; p < steps; ++p) {
        for (int i = 0; i < P->active[p]; ++i) {
            const int nbj = std::min(NB, n[P->order[i]] - NB * p);
            P->fl_diag[p] += 8.0 * nbj * nbj * nbj / 3.0;
        }
        const int u = P->upd[p];
        for (int k = 0; k < 3; ++k) {
            P->off[3 * p + k] = (int)P->sched.size();
            int64_t acc = 0;
            P->sched.push_back(0);
            for (int i = 0; i < u; ++i) {
                const int rest = n[P->order[i]] - NB * p - NB;
                int64_t c;
                if (k == 0) {
                    c = 2 * ceil_div(rest, NB);
                    P->fl_apply[p] += 8.0 * 2.0 * rest * NB * NB;
                } else if (k == 1) {
                    c = 0;  // (operand packing is done by the panel solve)
                } else {
                    c = sizeof(C) == sizeof(float2) ? (int64_t)(grp_rows_a(rest) / TC_BM) * (grp_rows_b(rest) / bn)
                                                    : (int64_t)ceil_div(rest, DM_BM) * ceil_div(rest, DM_BN);
                    P->fl_upd[p] += 8.0 * (double)rest * rest * NB;
                }
                acc += c;
                if (acc > 2000000000LL) return grim_fail(GRIM_ERR_ARGUMENT, "grouped factorization: too much work per step");
                P->sched.push_back((int)acc);
            }
            P->tot[3 * p + k] = (int)acc;
        }
    }
    return GRIM_OK;
}

// The launches of one grouped factorization, on h->stream (captured into a graph or not).
template <typename C>
static int grp_sequence(grim_context *h, const GrpPlan &P, const GrpSys *dsys, const int *dsched, int count,
                        int *dout, int *err) {
    const int steps = (int)P.active.size();
    const size_t tri = (size_t)(NB * NBP + NB) * sizeof(C);
    for (int p = 0; p < steps; ++p) {
        const int a = P.active[p], u = P.upd[p];
        k_grp_diag<C><<<a, 256, 0, h->stream>>>(dsys, p);
        GRIM_CHECK_LAUNCH_W(h, kname("k_grp_diag", sizeof(C)), P.fl_diag[p], 0);
        if (u > 0) {
            k_grp_apply<C><<<P.tot[3 * p], 256, tri, h->stream>>>(dsys, p, dsched + P.off[3 * p], u);
            GRIM_CHECK_LAUNCH_W(h, kname("k_grp_apply", sizeof(C)), P.fl_apply[p], 0);
        }
        if (a > u) {
            k_grp_last<C><<<a - u, 256, 0, h->stream>>>(dsys, p, u);
            GRIM_CHECK_LAUNCH(h, kname("k_grp_last", sizeof(C)));
        }
        if (u == 0) continue;
        if constexpr (sizeof(C) == sizeof(float2)) {
            // (the operands were packed by k_grp_apply)
            const int tiles = P.tot[3 * p + 2];
            if (grp_persistent() && P.bn == GRP_BN) {
                k_grp_tc_update_p<GRP_BN><<<std::min(tiles, h->sm_count), GRP_P_THREADS, GrpPCfg<GRP_BN>::SMEM_BYTES,
                                            h->stream>>>(dsys, p, dsched + P.off[3 * p + 2], u, tiles, err);
            } else if (grp_persistent()) {
                k_grp_tc_update_p<64><<<std::min(tiles, h->sm_count), GRP_P_THREADS, GrpPCfg<64>::SMEM_BYTES,
                                        h->stream>>>(dsys, p, dsched + P.off[3 * p + 2], u, tiles, err);
            } else if (P.bn == 64)
                k_grp_tc_update<64, 1><<<P.tot[3 * p + 2], TC_THREADS, TcCfg<64, 1, true>::SMEM_BYTES, h->stream>>>(
                    dsys, p, dsched + P.off[3 * p + 2], u, err);
            else
                k_grp_tc_update<GRP_BN, GRP_STAGES><<<P.tot[3 * p + 2], TC_THREADS,
                                                     TcCfg<GRP_BN, GRP_STAGES, true>::SMEM_BYTES, h->stream>>>(
                    dsys, p, dsched + P.off[3 * p + 2], u, err);
            GRIM_CHECK_LAUNCH_W(h, "k_grp_tc_update", P.fl_upd[p], 0);
        } else {
            k_grp_dmma_update<<<P.tot[3 * p + 2], DM_THREADS, DM_SMEM_BYTES, h->stream>>>(dsys, p,
                                                                                           dsched + P.off[3 * p + 2], u);
            GRIM_CHECK_LAUNCH_W(h, "k_grp_dmma_update", P.fl_upd[p], 0);
        }
    }
    k_grp_laswp<C><<<dim3(ceil_div(P.nmax, 128), count), 128, 0, h->stream>>>(dsys);
    GRIM_CHECK_LAUNCH(h, kname("k_grp_laswp", sizeof(C)));
    k_grp_flags<<<ceil_div(count, 128), 128, 0, h->stream>>>(dsys, count, dout);
    GRIM_CHECK_LAUNCH(h, "k_grp_flags");
    return GRIM_OK;
}

template <typename C>
static int grp_getrf(grim_context *h, int count, const int *n, void *const *A, const int64_t *lda, int *const *ipiv,
                     bool use_graph, int *info, int *pivoted) {
    GrpPlan P;
    GRIM_TRY(grp_plan<C>(count, n, grp_bn(), &P));
    static PerDeviceOnce attr;
    if (attr.needed()) {
        const int tri = (NB * NBP + NB) * (int)sizeof(C);
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_grp_apply<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri));
        if constexpr (sizeof(C) == sizeof(float2))
        {
            GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_grp_tc_update<GRP_BN, GRP_STAGES>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 TcCfg<GRP_BN, GRP_STAGES, true>::SMEM_BYTES));
            GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_grp_tc_update_p<GRP_BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 GrpPCfg<GRP_BN>::SMEM_BYTES));
            GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_grp_tc_update_p<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 GrpPCfg<64>::SMEM_BYTES));
            GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_grp_tc_update<64, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 TcCfg<64, 1, true>::SMEM_BYTES));
        }
        else
            GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_grp_dmma_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 DM_SMEM_BYTES));
        attr.mark();
    }
    // per-system device buffers, carved from one workspace at 256-byte boundaries
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t ws_bytes = 0, flag_ints = 0;
    for (int i = 0; i < count; ++i) {
        const int m = n[P.order[i]];
        ws_bytes += 2 * al((size_t)m * NB * sizeof(C));
        if (sizeof(C) == sizeof(float2) && m > NB)
            ws_bytes += 2 * al((size_t)grp_rows_a(m - NB) * GRP_KP * sizeof(float)) +
                        2 * al((size_t)grp_rows_b(m - NB) * GRP_KP * sizeof(float));
        flag_ints += 2 + 3 * (size_t)ceil_div(m, NB);
    }
    void *pws = nullptr, *pflags = nullptr, *ptab = nullptr, *psched = nullptr, *pout = nullptr;
    GRIM_TRY(grim_workspace(h, "grp_ws", ws_bytes, &pws));
    GRIM_TRY(grim_workspace(h, "grp_flags", flag_ints * sizeof(int), &pflags));
    GRIM_TRY(grim_workspace(h, "grp_table", (size_t)count * sizeof(GrpSys), &ptab));
    GRIM_TRY(grim_workspace(h, "grp_sched", P.sched.size() * sizeof(int), &psched));
    GRIM_TRY(grim_workspace(h, "grp_out", 2 * (size_t)count * sizeof(int), &pout));
    int *err = nullptr;
    if (sizeof(C) == sizeof(float2)) GRIM_TRY(tc_err_flag(h, &err));
    std::vector<GrpSys> tab(count);
    char *w = (char *)pws;
    int *f = (int *)pflags;
    for (int i = 0; i < count; ++i) {
        const int src = P.order[i], m = n[src];
        GrpSys &S = tab[i];
        S.A = A[src];
        S.lda = lda[src];
        S.n = m;
        S.npan = ceil_div(m, NB);
        S.ipiv = ipiv[src];
        S.bcol = w;
        w += al((size_t)m * NB * sizeof(C));
        S.brow = w;
        w += al((size_t)m * NB * sizeof(C));
        S.flags = f;
        f += 2 + 3 * S.npan;
        S.pa_hi = S.pa_lo = S.pb_hi = S.pb_lo = nullptr;
        S.static_pivot = h->pivot_mode == GRIM_PIVOT_STATIC;
        if (sizeof(C) == sizeof(float2) && m > NB) {
            const size_t ra = (size_t)grp_rows_a(m - NB) * GRP_KP, rb = (size_t)grp_rows_b(m - NB) * GRP_KP;
            S.pa_hi = (float *)w;
            w += al(ra * sizeof(float));
            S.pa_lo = (float *)w;
            w += al(ra * sizeof(float));
            S.pb_hi = (float *)w;
            w += al(rb * sizeof(float));
            S.pb_lo = (float *)w;
            w += al(rb * sizeof(float));
        }
    }
    GRIM_CHECK_CUDA(cudaMemcpyAsync(ptab, tab.data(), (size_t)count * sizeof(GrpSys), cudaMemcpyHostToDevice, h->stream));
    GRIM_CHECK_CUDA(cudaMemcpyAsync(psched, P.sched.data(), P.sched.size() * sizeof(int), cudaMemcpyHostToDevice,
                                    h->stream));
    GRIM_CHECK_CUDA(cudaMemsetAsync(pflags, 0, flag_ints * sizeof(int), h->stream));
    const GrpSys *dsys = (const GrpSys *)ptab;
    const int *dsched = (const int *)psched;
    int *dout = (int *)pout;
    if (use_graph && !h->profiling) {
        std::vector<int64_t> key = {(int64_t)sizeof(C), (int64_t)P.bn, (int64_t)grp_persistent(), (int64_t)count,
                                    (int64_t)(intptr_t)pws,
                                    (int64_t)(intptr_t)pflags, (int64_t)(intptr_t)ptab, (int64_t)(intptr_t)psched,
                                    (int64_t)(intptr_t)pout, (int64_t)(intptr_t)err};
        for (int i = 0; i < count; ++i) key.push_back(n[P.order[i]]);
        if (!h->grp_exec || key != h->grp_key) {
            if (h->grp_exec) {
                cudaGraphExecDestroy(h->grp_exec);
                h->grp_exec = nullptr;
                h->grp_key.clear();
            }
            // captured on the handle's private stream (the caller's may be the legacy
            // default stream, which cannot be captured), launched on the caller's
            GRIM_TRY(lookahead_streams(h, 2));
            const cudaStream_t caller = h->stream;
            GRIM_CHECK_CUDA(cudaStreamBeginCapture(h->chain, cudaStreamCaptureModeThreadLocal));
            const int64_t l0 = h->launches;
            h->stream = h->chain;
            const int st = grp_sequence<C>(h, P, dsys, dsched, count, dout, err);
            h->stream = caller;
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(h->chain, &graph);
            if (st != GRIM_OK) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            GRIM_CHECK_CUDA(ce);
            const cudaError_t ie = cudaGraphInstantiate(&h->grp_exec, graph, 0);
            cudaGraphDestroy(graph);
            GRIM_CHECK_CUDA(ie);
            h->grp_key = key;
            h->grp_graph_launches = h->launches - l0;
            h->launches = l0;
        }
        GRIM_CHECK_CUDA(cudaGraphLaunch(h->grp_exec, h->stream));
        h->launches += h->grp_graph_launches;
    } else {
        GRIM_TRY(grp_sequence<C>(h, P, dsys, dsched, count, dout, err));
    }
    std::vector<int> out(2 * (size_t)count);
    GRIM_CHECK_CUDA(cudaMemcpyAsync(out.data(), dout, out.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    if (sizeof(C) == sizeof(float2)) GRIM_TRY(tc_err_check(h, "grouped factorization"));
    for (int i = 0; i < count; ++i) {
        if (info) info[P.order[i]] = out[2 * i];
        if (pivoted) pivoted[P.order[i]] = out[2 * i + 1];
    }
    return GRIM_OK;
}

extern "C" int grim_getrf_grouped(grim_handle_t h, int count, const int *n, void *const *A, const int64_t *lda,
                                  int *const *ipiv, int complex64, int use_graph, int *info, int *pivoted) {
    if (!h || count <= 0 || count > 65535 || !n || !A || !lda || !ipiv || !info)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_getrf_grouped: bad arguments");
    for (int i = 0; i < count; ++i)
        if (n[i] <= 0 || !A[i] || !ipiv[i] || lda[i] < n[i])
            return grim_fail(GRIM_ERR_ARGUMENT, "grim_getrf_grouped: bad system " + std::to_string(i));
    DeviceGuard g(h->device);
    if (complex64) return grp_getrf<float2>(h, count, n, A, lda, ipiv, use_graph != 0, info, pivoted);
    return grp_getrf<double2>(h, count, n, A, lda, ipiv, use_graph != 0, info, pivoted);
}

// Refinement against an existing complex64 factorization with the stopping test chosen
// by precision_mode (GRIM_PREC_MIXED: relative residual, GRIM_PREC_MIXED_BERR: backward
// error).
extern "C" int grim_zgesv_refine_factored(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda,
                                          const void *A32, int64_t lda32, void *LU32, const int *ipiv, void *B,
                                          int64_t ldb, int precision_mode, double tol, int max_iter,
                                          grim_solve_info *stats) {
    if (!h || n <= 0 || nrhs <= 0 || !B || ldb < n || (!A && !A32) || (A && lda < n) || (A32 && lda32 < n) || !LU32 ||
        !ipiv || (precision_mode != GRIM_PREC_MIXED && precision_mode != GRIM_PREC_MIXED_BERR))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_zgesv_refine_factored: bad arguments");
    DeviceGuard g(h->device);
    grim_solve_info st{};
    st.precision_mode = precision_mode;
    const bool berr_test = precision_mode == GRIM_PREC_MIXED_BERR;
    StreamTimer ts(h->stream);
    int s;
    if (A)
        s = mixed_refine<double2>(h, n, nrhs, (const double2 *)A, lda, (float2 *)LU32, ipiv, (double2 *)B, ldb, tol,
                                  max_iter, &st, berr_test);
    else
        s = mixed_refine<float2>(h, n, nrhs, (const float2 *)A32, lda32, (float2 *)LU32, ipiv, (double2 *)B, ldb, tol,
                                 max_iter, &st, berr_test);
    st.ms_solve = ts.stop_ms();
    h->last = st;
    if (stats) *stats = st;
    return s;
}

// ============================================================== Galerkin far blocks (boundary B2)
// Argument check of twod/assembly/native/far.c:114-117 (status 3).
static bool far_args_ok(int64_t mb, int64_t nb, int q, int width, int want_s, int want_k, int mirrored,
                        int intervals, int degree, const void *acc_s, const void *acc_k, const void *acc_kt) {
    return !(mb < 0 || nb < 0 || q < 1 || width < 1 || width > FAR_MAX_WIDTH || intervals < 1 || degree < 0 ||
             degree > 32 || (!want_s && !want_k) || (want_s && !acc_s) || (want_k && !acc_k) ||
             (want_k && mirrored && !acc_kt));
}

// Device-pointer form: returns 0, 2 (a far distance below the table: the caller's
// fallback case, accumulators undefined) or 3 (bad arguments); GRIM_ERR_CUDA on a device
// error.
extern "C" int grim_far_block(grim_handle_t h, int64_t mb, int64_t nb, int q, int width, const double *obs_pts,
                              const double *src_pts, const double *qw, const double *phi, const double *obs_norm,
                              const double *src_norm, const uint8_t *far, int obs_normal_deriv, int want_s,
                              int want_k, int mirrored, double k_re, double k_im, int intervals,
                              const double *bounds, int degree, const double *coeff, double *acc_s, double *acc_k,
                              double *acc_kt) {
    if (!h) return grim_fail(GRIM_ERR_ARGUMENT, "grim_far_block: null handle");
    if (!far_args_ok(mb, nb, q, width, want_s, want_k, mirrored, intervals, degree, acc_s, acc_k, acc_kt)) {
        grim_set_error("grim_far_block: bad arguments");
        return 3;
    }
    if (mb == 0 || nb == 0) return GRIM_OK;
    DeviceGuard g(h->device);
    void *pst = nullptr;
    GRIM_TRY(grim_workspace(h, "far_status", sizeof(int), &pst));
    int *status = (int *)pst;
    GRIM_CHECK_CUDA(cudaMemsetAsync(status, 0, sizeof(int), h->stream));
    const FarTable t{intervals, degree, bounds, coeff, k_re, k_im, ((uintptr_t)coeff & 15) == 0};
    const int64_t pairs = mb * nb;
    const int threads = 128;
    const int64_t blocks = (pairs + threads - 1) / threads;
    if (blocks > 2147483647LL) {
        grim_set_error("grim_far_block: too many pairs for one launch");
        return 3;
    }
    const size_t smem = intervals + 1 <= FAR_SMEM_BOUNDS ? (size_t)(intervals + 1) * sizeof(double) : 0;
    static PerDeviceOnce attr;
    if (attr.needed()) {
        const int mx = FAR_SMEM_BOUNDS * (int)sizeof(double);
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_far_block<0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_far_block<2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_far_block<3, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
        GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_far_block<4, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
        attr.mark();
    }
#define FAR_LAUNCH(W, MINB)                                                                                      \
    k_far_block<W, MINB><<<(unsigned)blocks, threads, smem, h->stream>>>(mb, nb, q, width, obs_pts, src_pts, qw, phi, \
                                                                obs_norm, src_norm, far, obs_normal_deriv,       \
                                                                want_s, want_k, mirrored, t, acc_s, acc_k,       \
                                                                acc_kt, status)
    if (width == 2) FAR_LAUNCH(2, 4);
    else if (width == 3) FAR_LAUNCH(3, 2);
    else if (width == 4) FAR_LAUNCH(4, 1);
    else FAR_LAUNCH(0, 1);
#undef FAR_LAUNCH
    GRIM_CHECK_LAUNCH_W(h, "k_far_block", 0.0, 0.0);
    int hs = 0;
    GRIM_CHECK_CUDA(cudaMemcpyAsync(&hs, status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return hs ? 2 : GRIM_OK;
}

// Host-buffer form with the exact signature and status codes of the reference's
// ghost_far_block (twod/assembly/native/far.c:193-207, loaded by
// twod/assembly/native/far.py:184-199): copies in, runs grim_far_block on the calling
// thread's own handle (current device), copies the accumulators back.  Thread-safe.
extern "C" int ghost_far_block(int64_t mb, int64_t nb, int q, int width, const double *obs_pts,
                               const double *src_pts, const double *qw, const double *phi, const double *obs_norm,
                               const double *src_norm, const uint8_t *far, int obs_normal_deriv, int want_s,
                               int want_k, int mirrored, double k_re, double k_im, int intervals,
                               const double *bounds, int degree, const double *coeff, double *acc_s, double *acc_k,
                               double *acc_kt) {
    if (!far_args_ok(mb, nb, q, width, want_s, want_k, mirrored, intervals, degree, acc_s, acc_k, acc_kt)) return 3;
    if (mb == 0 || nb == 0) return 0;
    static thread_local grim_context *h = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GRIM_ERR_CUDA;
    if (!h || h->device != dev) {
        if (h) grim_destroy(h);
        h = nullptr;
        GRIM_TRY(grim_create(dev, &h));
    }
    DeviceGuard g(h->device);
    const bool with_kt = want_k && mirrored;
    const size_t acc_bytes = (size_t)width * width * mb * nb * 2 * sizeof(double);
    const size_t pts_o = (size_t)mb * q * 2, pts_s = (size_t)nb * q * 2;
    const size_t tab_c = (size_t)intervals * (degree + 1) * 4;
    size_t dbl = pts_o + pts_s + q + (size_t)q * width + 2 * (size_t)mb + 2 * (size_t)nb + (intervals + 1) + tab_c;
    const size_t bytes = dbl * sizeof(double) + (size_t)mb * nb + 3 * acc_bytes + 1024;
    void *pw = nullptr;
    GRIM_TRY(grim_workspace(h, "far_io", bytes, &pw));
    double *d = (double *)pw;
    double *d_op = d, *d_sp = d_op + pts_o, *d_qw = d_sp + pts_s, *d_phi = d_qw + q, *d_on = d_phi + (size_t)q * width,
           *d_sn = d_on + 2 * mb, *d_b = d_sn + 2 * nb;
    double *d_c = (double *)(((uintptr_t)(d_b + (intervals + 1)) + 15) & ~(uintptr_t)15);  // 16-byte aligned
    double *d_as = (double *)(((uintptr_t)(d_c + tab_c) + 255) & ~(uintptr_t)255);
    double *d_ak = (double *)((char *)d_as + acc_bytes), *d_akt = (double *)((char *)d_ak + acc_bytes);
    uint8_t *d_far = (uint8_t *)((char *)d_akt + acc_bytes);
    auto up = [&](void *dst, const void *src, size_t n) {
        return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, h->stream);
    };
    GRIM_CHECK_CUDA(up(d_op, obs_pts, pts_o * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_sp, src_pts, pts_s * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_qw, qw, q * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_phi, phi, (size_t)q * width * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_on, obs_norm, 2 * mb * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_sn, src_norm, 2 * nb * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_b, bounds, (intervals + 1) * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_c, coeff, tab_c * sizeof(double)));
    GRIM_CHECK_CUDA(up(d_far, far, (size_t)mb * nb));
    if (want_s) GRIM_CHECK_CUDA(up(d_as, acc_s, acc_bytes));
    if (want_k) GRIM_CHECK_CUDA(up(d_ak, acc_k, acc_bytes));
    if (with_kt) GRIM_CHECK_CUDA(up(d_akt, acc_kt, acc_bytes));
    const int s = grim_far_block(h, mb, nb, q, width, d_op, d_sp, d_qw, d_phi, d_on, d_sn, d_far, obs_normal_deriv,
                                 want_s, want_k, mirrored, k_re, k_im, intervals, d_b, degree, d_c,
                                 want_s ? d_as : nullptr, want_k ? d_ak : nullptr, with_kt ? d_akt : nullptr);
    if (s != GRIM_OK) return s;
    auto down = [&](void *dst, const void *src, size_t n) {
        return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, h->stream);
    };
    if (want_s) GRIM_CHECK_CUDA(down(acc_s, d_as, acc_bytes));
    if (want_k) GRIM_CHECK_CUDA(down(acc_k, d_ak, acc_bytes));
    if (with_kt) GRIM_CHECK_CUDA(down(acc_kt, d_akt, acc_bytes));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

// B1 drop-in with host buffers.
extern "C" int grim_zgesv_batched(grim_handle_t h, int n, int nrhs, const double *A, int lda, double *B, int ldb,
                                  int precision_mode, int *info) {
    if (!h || n <= 0 || nrhs <= 0 || !A || !B || lda < n || ldb < n)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_zgesv_batched: bad arguments");
    DeviceGuard g(h->device);
    void *pa = nullptr, *pb = nullptr;
    GRIM_TRY(grim_workspace(h, "h_A", (size_t)n * n * sizeof(double2), &pa));
    GRIM_TRY(grim_workspace(h, "h_B", (size_t)n * nrhs * sizeof(double2), &pb));
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(pa, n * sizeof(double2), A, (size_t)lda * sizeof(double2), n * sizeof(double2), n,
                                      cudaMemcpyHostToDevice, h->stream));
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(pb, n * sizeof(double2), B, (size_t)ldb * sizeof(double2), n * sizeof(double2),
                                      nrhs, cudaMemcpyHostToDevice, h->stream));
    int s = grim_zgesv_mixed(h, n, nrhs, pa, n, nullptr, 0, pb, n, precision_mode, 2e-12, 10, info, nullptr);
    if (s != GRIM_OK) return s;
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(double2), pb, n * sizeof(double2), n * sizeof(double2),
                                      nrhs, cudaMemcpyDeviceToHost, h->stream));
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return GRIM_OK;
}

// ============================================================== profiling
void grim_prof_mark(grim_context *h, const char *name, double flops, double bytes) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, h->stream);
    h->marks.push_back({std::string(name), e, flops, bytes});
}

static void prof_clear(grim_context *h) {
    for (auto &m : h->marks) cudaEventDestroy(m.ev);
    h->marks.clear();
    if (h->prof_start) {
        cudaEventDestroy(h->prof_start);
        h->prof_start = nullptr;
    }
}

extern "C" int grim_profile_enable(grim_handle_t h, int enable) {
    if (!h) return grim_fail(GRIM_ERR_ARGUMENT, "null handle");
    DeviceGuard g(h->device);
    prof_clear(h);
    h->profiling = enable ? 1 : 0;
    if (enable) {
        GRIM_CHECK_CUDA(cudaEventCreate(&h->prof_start));
        GRIM_CHECK_CUDA(cudaEventRecord(h->prof_start, h->stream));
    }
    return GRIM_OK;
}

// JSON object {"kernel": {"launches": n, "ms": total, "flops": f, "bytes": b}, ...}; each
// kernel's time is the span from the previous event on the stream to its end event.
extern "C" int grim_profile_report(grim_handle_t h, char *buf, int len) {
    if (!h || !buf || len <= 0) return grim_fail(GRIM_ERR_ARGUMENT, "grim_profile_report: bad arguments");
    DeviceGuard g(h->device);
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    struct Agg { int n = 0; double ms = 0, flops = 0, bytes = 0; };
    std::vector<std::pair<std::string, Agg>> agg;
    cudaEvent_t prev = h->prof_start;
    for (auto &m : h->marks) {
        float ms = 0.f;
        if (prev) cudaEventElapsedTime(&ms, prev, m.ev);
        prev = m.ev;
        auto it = std::find_if(agg.begin(), agg.end(), [&](const std::pair<std::string, Agg> &p) { return p.first == m.name; });
        if (it == agg.end()) { agg.push_back({m.name, Agg()}); it = agg.end() - 1; }
        it->second.n++;
        it->second.ms += ms;
        it->second.flops += m.flops;
        it->second.bytes += m.bytes;
    }
    std::string out = "{";
    for (size_t i = 0; i < agg.size(); ++i) {
        char tmp[256];
        std::snprintf(tmp, sizeof(tmp), "%s\"%s\": {\"launches\": %d, \"ms\": %.6f, \"flops\": %.6e, \"bytes\": %.6e}",
                      i ? ", " : "", agg[i].first.c_str(), agg[i].second.n, agg[i].second.ms, agg[i].second.flops,
                      agg[i].second.bytes);
        out += tmp;
    }
    out += "}";
    if ((int)out.size() + 1 > len) return grim_fail(GRIM_ERR_ARGUMENT, "grim_profile_report: buffer too small");
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return GRIM_OK;
}

// ============================================================== body of revolution
extern "C" int64_t grim_bor_moments_size(int ne, int mmax) {
    return (int64_t)ne * ne * (mmax + 2) * BOR_SLOTS * (int64_t)sizeof(double2);
}

extern "C" int64_t grim_bor_mfie_moments_size(int ne, int mmax) {
    return (int64_t)ne * ne * (mmax + 2) * BOR_KSLOTS * (int64_t)sizeof(double2);
}

template <bool MFIE>
static size_t bor_tail_smem(int nm) {
    const int NV = MFIE ? 5 : 1, nsl = MFIE ? BOR_ALL_SLOTS : BOR_SLOTS, S = BOR_THREADS / nm;
    return sizeof(double2) * ((size_t)S * nm * NV + (size_t)nm * NV + (size_t)nm * nsl) + sizeof(double) * nsl;
}

template <bool MFIE>
static int bor_moments_launch(grim_context *h, int ne, const double *nodes, const unsigned char *d_cls, double k,
                              int mmax, int nxi_cap, const std::vector<BorItem> &items,
                              const std::vector<int4> &pairs, const double *d_rule, double2 *mom, double2 *momk) {
    const int nm = mmax + 2, NV = MFIE ? 5 : 1, nsl = MFIE ? BOR_ALL_SLOTS : BOR_SLOTS;
    // far pairs
    const int S = BOR_THREADS / nm, NPP = BOR_FAR_ORDER * BOR_FAR_ORDER;
    const size_t far_smem = sizeof(double2) * ((size_t)NV * BOR_FAR_CHUNK + (size_t)S * nm * NV + (size_t)NPP * nm * NV) +
                            sizeof(double) * NPP * nsl;
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_bor_far<MFIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)far_smem));
    k_bor_far<MFIE><<<dim3(ne, ne), BOR_THREADS, far_smem, h->stream>>>(ne, nodes, d_cls, k, mmax, nxi_cap, mom,
                                                                          momk);
    GRIM_CHECK_LAUNCH(h, MFIE ? "k_bor_far<cfie>" : "k_bor_far<efie>");
    if (items.empty()) return GRIM_OK;
    void *p_items = nullptr, *p_pairs = nullptr, *p_part = nullptr;
    GRIM_TRY(grim_workspace(h, "bor_items", items.size() * sizeof(BorItem), &p_items));
    GRIM_TRY(grim_workspace(h, "bor_pairs", pairs.size() * sizeof(int4), &p_pairs));
    GRIM_TRY(grim_workspace(h, "bor_part", items.size() * (size_t)nm * nsl * sizeof(double2), &p_part));
    GRIM_CHECK_CUDA(cudaMemcpyAsync(p_items, items.data(), items.size() * sizeof(BorItem), cudaMemcpyHostToDevice,
                                    h->stream));
    GRIM_CHECK_CUDA(cudaMemcpyAsync(p_pairs, pairs.data(), pairs.size() * sizeof(int4), cudaMemcpyHostToDevice,
                                    h->stream));
    const int chr = nm <= 64 ? 64 : 32;
    // rows and the groups' partial sums share one region (red = S nm NV complex)
    const size_t near_smem = sizeof(double2) * ((size_t)(NV + 2) * BOR_NEAR_EVAL +
                                                std::max((size_t)chr * (nm | 1), (size_t)S * nm * NV)) +
                             bor_tail_smem<MFIE>(nm) - sizeof(double2) * (size_t)S * nm * NV;
    GRIM_CHECK_CUDA(cudaFuncSetAttribute(k_bor_near<MFIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)near_smem));
    k_bor_near<MFIE><<<(unsigned)items.size(), BOR_THREADS, near_smem, h->stream>>>(
        (const BorItem *)p_items, nodes, d_rule, k, mmax, chr, (double2 *)p_part);
    GRIM_CHECK_LAUNCH(h, MFIE ? "k_bor_near<cfie>" : "k_bor_near<efie>");
    k_bor_near_reduce<MFIE><<<(unsigned)pairs.size(), 256, 0, h->stream>>>(ne, mmax, (const int4 *)p_pairs,
                                                                           (const double2 *)p_part, mom, momk);
    GRIM_CHECK_LAUNCH(h, "k_bor_near_reduce");
    return GRIM_OK;
}

extern "C" int grim_bor_moments(grim_handle_t h, int ne, const double *nodes, double k, int mmax, int nxi_max,
                                const unsigned char *pair_class, int n_rule, const double *rule,
                                const int *rule_start, void *mom, void *mom_k) {
    if (!h || ne < 2 || !nodes || !mom || !(k > 0) || mmax < 0 || mmax + 2 > BOR_MAX_MODES || nxi_max < 32 ||
        nxi_max > BOR_MAX_NXI || ne > 65535 || !pair_class || n_rule <= 0 || !rule || !rule_start)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_moments: bad arguments");
    // rule_start[0..4]: point ranges of the self (diagonal), adjacent f = e + 1, adjacent
    // f = e - 1 and regular near rules in `rule` (s, s', w per point pair)
    for (int i = 0; i < 4; ++i)
        if (rule_start[i] < 0 || rule_start[i] >= rule_start[i + 1] || rule_start[i + 1] > n_rule)
            return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_moments: bad rule ranges");
    std::vector<BorItem> items;
    std::vector<int4> pairs;
    for (int e = 0; e < ne; ++e)
        for (int f = 0; f < ne; ++f) {
            const unsigned char c = pair_class[(size_t)e * ne + f];
            if (c > 2) return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_moments: pair class must be 0, 1 or 2");
            if (c == 1 && std::abs(e - f) > 1)
                return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_moments: class 1 is for self and adjacent pairs");
            if (c == 0) continue;
            const int kind = c == 2 ? 3 : (e == f ? 0 : (f == e + 1 ? 1 : 2));
            const int first = (int)items.size();
            for (int r = rule_start[kind]; r < rule_start[kind + 1]; r += BOR_NEAR_CHUNK)
                items.push_back(BorItem{e, f, r, std::min(r + BOR_NEAR_CHUNK, rule_start[kind + 1])});
            pairs.push_back(make_int4(e, f, first, (int)items.size()));
        }
    DeviceGuard g(h->device);
    void *p_cls = nullptr, *p_rule = nullptr;
    GRIM_TRY(grim_workspace(h, "bor_cls", (size_t)ne * ne, &p_cls));
    GRIM_TRY(grim_workspace(h, "bor_rule", (size_t)3 * n_rule * sizeof(double), &p_rule));
    GRIM_CHECK_CUDA(cudaMemcpyAsync(p_cls, pair_class, (size_t)ne * ne, cudaMemcpyHostToDevice, h->stream));
    GRIM_CHECK_CUDA(cudaMemcpyAsync(p_rule, rule, (size_t)3 * n_rule * sizeof(double), cudaMemcpyHostToDevice,
                                    h->stream));
    // per-launch profiling: the kernels' spans start here, not at the caller's host work
    if (h->profiling) grim_prof_mark(h, "bor_upload", 0, 0);
    // a multiple of 32 keeps the shared-memory sections after the sample table 16-byte aligned
    const int cap = std::min(BOR_MAX_NXI, (std::max(32, nxi_max) + 31) / 32 * 32);
    int s;
    if (mom_k)
        s = bor_moments_launch<true>(h, ne, nodes, (const unsigned char *)p_cls, k, mmax, cap, items, pairs,
                                     (const double *)p_rule, (double2 *)mom, (double2 *)mom_k);
    else
        s = bor_moments_launch<false>(h, ne, nodes, (const unsigned char *)p_cls, k, mmax, cap, items, pairs,
                                      (const double *)p_rule, (double2 *)mom, nullptr);
    GRIM_TRY(s);
    // the host vectors above are freed on return: wait for the uploads that read them
    GRIM_CHECK_CUDA(cudaStreamSynchronize(h->stream));
    return GRIM_OK;
}

extern "C" int grim_bor_assemble(grim_handle_t h, int ne, const double *nodes, double k, int mmax, int m,
                                 const void *mom, const void *mom_k, double alpha, int nred, const int *red_full,
                                 const void *red_w, void *Z, int64_t ldz) {
    if (!h || ne < 2 || !nodes || !mom || !red_full || !red_w || !Z || nred <= 0 || ldz < nred || abs(m) > mmax ||
        !(alpha >= 0.0 && alpha <= 1.0) || (!mom_k && alpha != 1.0))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_assemble: bad arguments");
    DeviceGuard g(h->device);
    dim3 grid(ceil_div(nred, 16), ceil_div(nred, 16)), block(16, 16);
    k_bor_assemble<<<grid, block, 0, h->stream>>>(ne, mmax, m, k, (const double2 *)mom, (const double2 *)mom_k, alpha,
                                                  nred, red_full, (const double2 *)red_w, nodes, (double2 *)Z, ldz);
    GRIM_CHECK_LAUNCH(h, "k_bor_assemble");
    return GRIM_OK;
}

extern "C" int grim_bor_excitation(grim_handle_t h, int ne, const double *nodes, double k, int m, int nth,
                                   const double *thetas_deg, int far, double alpha, int nred, const int *red_full,
                                   const void *red_w, void *V, int64_t ldv) {
    if (!h || ne < 2 || !nodes || !thetas_deg || !red_full || !red_w || !V || nth <= 0 || 2 * nth > 65535 ||
        nred <= 0 || ldv < nred || !(alpha >= 0.0 && alpha <= 1.0))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_excitation: bad arguments");
    DeviceGuard g(h->device);
    void *p_tab = nullptr;
    // sized in steps of 512 aspects so that a handle rarely regrows it between requests
    GRIM_TRY(grim_workspace(h, "bor_bessel", (size_t)5 * BOR_FAR_ORDER * ne * (size_t)(ceil_div(nth, 512) * 512) *
                                                 sizeof(double), &p_tab));
    k_bor_bessel<<<dim3(ceil_div(BOR_FAR_ORDER * ne, 128), nth), 128, 0, h->stream>>>(ne, nodes, k, m, nth, thetas_deg,
                                                                                      (double *)p_tab);
    GRIM_CHECK_LAUNCH(h, "k_bor_bessel");
    dim3 grid(ceil_div(nred, 128), 2 * nth);
    k_bor_excitation<<<grid, 128, 0, h->stream>>>(ne, nodes, m, nth, thetas_deg, (const double *)p_tab, far, alpha,
                                                  nred, red_full, (const double2 *)red_w, (double2 *)V, ldv);
    GRIM_CHECK_LAUNCH(h, "k_bor_excitation");
    return GRIM_OK;
}

extern "C" int grim_bor_farfield_accumulate(grim_handle_t h, int nred, int ncol, const void *W, int64_t ldw,
                                            const void *X, int64_t ldx, void *amp) {
    if (!h || nred <= 0 || ncol <= 0 || !W || !X || !amp || ldw < nred || ldx < nred)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_farfield_accumulate: bad arguments");
    DeviceGuard g(h->device);
    k_bor_farfield_accumulate<<<ncol, 256, 0, h->stream>>>(nred, ncol, (const double2 *)W, ldw, (const double2 *)X,
                                                           ldx, (double2 *)amp);
    GRIM_CHECK_LAUNCH(h, "k_bor_farfield_accumulate");
    return GRIM_OK;
}

// ---- mirror halves (reference bor/factor.py:37 MirrorSplit)
static bool mirror_args_ok(int k, const int *p1, const int *p2, const double *s, int nfe, const int *fe, int nfo,
                           const int *fo) {
    return k >= 0 && nfe >= 0 && nfo >= 0 && k + nfe > 0 && k + nfo > 0 && (k == 0 || (p1 && p2 && s)) &&
           (nfe == 0 || fe) && (nfo == 0 || fo);
}

extern "C" int grim_bor_mirror_halves(grim_handle_t h, int n, const void *Z, int64_t ldz, int k, const int *p1,
                                      const int *p2, const double *s, int nfe, const int *fe, int nfo, const int *fo,
                                      void *He, void *Ho) {
    if (!h || n <= 0 || !Z || ldz < n || !He || !Ho || 2 * k + nfe + nfo != n ||
        !mirror_args_ok(k, p1, p2, s, nfe, fe, nfo, fo))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_mirror_halves: bad arguments");
    DeviceGuard g(h->device);
    const BorMirror mr{k, nfe, nfo, p1, p2, fe, fo, s};
    const int m = k + std::max(nfe, nfo);
    k_bor_mirror_halves<<<dim3(ceil_div(m, 16), ceil_div(m, 16)), dim3(16, 16), 0, h->stream>>>(
        mr, (const double2 *)Z, ldz, (double2 *)He, (double2 *)Ho);
    GRIM_CHECK_LAUNCH(h, "k_bor_mirror_halves");
    return GRIM_OK;
}

extern "C" int grim_bor_mirror_asymmetry(grim_handle_t h, int n, const void *Z, int64_t ldz, const int *target,
                                         const double *sign, double *out) {
    if (!h || n <= 0 || !Z || ldz < n || !target || !sign || !out)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_mirror_asymmetry: bad arguments");
    DeviceGuard g(h->device);
    GRIM_CHECK_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(double), h->stream));
    k_bor_mirror_asym<<<dim3(ceil_div(n, 16), ceil_div(n, 16)), dim3(16, 16), 0, h->stream>>>(
        n, (const double2 *)Z, ldz, target, sign, (unsigned long long *)out);
    GRIM_CHECK_LAUNCH(h, "k_bor_mirror_asym");
    return GRIM_OK;
}

extern "C" int grim_bor_mirror_split(grim_handle_t h, int nrhs, const void *B, int64_t ldb, int k, const int *p1,
                                     const int *p2, const double *s, int nfe, const int *fe, int nfo, const int *fo,
                                     void *Be, void *Bo) {
    if (!h || nrhs <= 0 || nrhs > 65535 || !B || ldb < 2 * k + nfe + nfo || !Be || !Bo ||
        !mirror_args_ok(k, p1, p2, s, nfe, fe, nfo, fo))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_mirror_split: bad arguments");
    DeviceGuard g(h->device);
    const BorMirror mr{k, nfe, nfo, p1, p2, fe, fo, s};
    const int m = k + std::max(nfe, nfo);
    k_bor_mirror_split<<<dim3(ceil_div(m, 128), nrhs), 128, 0, h->stream>>>(mr, nrhs, (const double2 *)B, ldb,
                                                                             (double2 *)Be, (double2 *)Bo);
    GRIM_CHECK_LAUNCH(h, "k_bor_mirror_split");
    return GRIM_OK;
}

extern "C" int grim_bor_mirror_join(grim_handle_t h, int nrhs, const void *Ye, const void *Yo, int k, const int *p1,
                                    const int *p2, const double *s, int nfe, const int *fe, int nfo, const int *fo,
                                    void *X, int64_t ldx) {
    if (!h || nrhs <= 0 || nrhs > 65535 || !Ye || !Yo || !X || ldx < 2 * k + nfe + nfo ||
        !mirror_args_ok(k, p1, p2, s, nfe, fe, nfo, fo))
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_bor_mirror_join: bad arguments");
    DeviceGuard g(h->device);
    const BorMirror mr{k, nfe, nfo, p1, p2, fe, fo, s};
    const int m = k + std::max(nfe, nfo);
    k_bor_mirror_join<<<dim3(ceil_div(m, 128), nrhs), 128, 0, h->stream>>>(mr, nrhs, (const double2 *)Ye,
                                                                            (const double2 *)Yo, (double2 *)X, ldx);
    GRIM_CHECK_LAUNCH(h, "k_bor_mirror_join");
    return GRIM_OK;
}

// ============================================================== allocation-free backward error
#include "noalloc.cu"
