// Elementwise conversions, residual norms and backward errors for the dense solves.
#pragma once
#include "common.cuh"

// ------------------------------------------------------------------ elementwise / norms
template <typename TO, typename TI>
__global__ void k_convert(int m, int ncol, const TI *__restrict__ src, int64_t lds, TO *__restrict__ dst, int64_t ldd) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= m || c >= ncol) return;
    const TI v = src[(int64_t)c * lds + r];
    TO w;
    w.x = (decltype(w.x))v.x;
    w.y = (decltype(w.y))v.y;
    dst[(int64_t)c * ldd + r] = w;
}

// X += D (D complex64 or complex128)
template <typename TD>
__global__ void k_add_update(int m, int ncol, double2 *X, int64_t ldx, const TD *__restrict__ D, int64_t ldd) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= m || c >= ncol) return;
    const TD d = D[(int64_t)c * ldd + r];
    double2 &x = X[(int64_t)c * ldx + r];
    x.x += (double)d.x;
    x.y += (double)d.y;
}

// Row sums of |A_ij| (modulus) in two passes: partial[ch][r] over the column chunk ch
// (grid = row tiles x ROWSUM_CHUNKS, coalesced along rows), then a fixed-order sum.
#define ROWSUM_CHUNKS 64
template <typename TA>
__global__ void k_row_abs_partial(int n, const TA *__restrict__ A, int64_t lda, double *partial) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int ch = blockIdx.y;
    if (r >= n) return;
    const int per = (n + ROWSUM_CHUNKS - 1) / ROWSUM_CHUNKS;
    const int c0 = ch * per, c1 = min(n, c0 + per);
    double s = 0.0;
    for (int c = c0; c < c1; ++c) {
        const TA v = A[(int64_t)c * lda + r];
        s += hypot((double)v.x, (double)v.y);
    }
    partial[(int64_t)ch * n + r] = s;
}

__global__ void k_row_abs_finish(int n, const double *partial, double *rowsum) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    double s = 0.0;
    for (int ch = 0; ch < ROWSUM_CHUNKS; ++ch) s += partial[(int64_t)ch * n + r];
    rowsum[r] = s;
}

__global__ void k_max_reduce(int n, const double *v, double *out) {
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, v[i]);
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    __shared__ double w[32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? w[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
        if (threadIdx.x == 0) *out = m;
    }
}

// Per-column max modulus of up to three column blocks (R, X, B) -> out[3*ncol].
// max that propagates NaN (fmax drops it): a non-finite residual or solution must not
// read as a small backward error.
__device__ __forceinline__ double max_nan(double a, double b) { return (a > b || a != a) ? a : b; }

template <typename TX>
__global__ void k_col_absmax3(int m, const double2 *R, int64_t ldr, const TX *X, int64_t ldx, const double2 *B,
                              int64_t ldb, double *out) {
    const int c = blockIdx.x;
    double mr = 0.0, mx = 0.0, mb = 0.0;
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
        const double2 a = R[(int64_t)c * ldr + r];
        const TX x = X[(int64_t)c * ldx + r];
        const double2 b = B[(int64_t)c * ldb + r];
        mr = max_nan(mr, hypot(a.x, a.y));
        mx = max_nan(mx, hypot((double)x.x, (double)x.y));
        mb = max_nan(mb, hypot(b.x, b.y));
    }
    for (int off = 16; off > 0; off >>= 1) {
        mr = max_nan(mr, __shfl_down_sync(0xffffffffu, mr, off));
        mx = max_nan(mx, __shfl_down_sync(0xffffffffu, mx, off));
        mb = max_nan(mb, __shfl_down_sync(0xffffffffu, mb, off));
    }
    __shared__ double w[3][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { w[0][warp] = mr; w[1][warp] = mx; w[2][warp] = mb; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        mr = lane < nw ? w[0][lane] : 0.0;
        mx = lane < nw ? w[1][lane] : 0.0;
        mb = lane < nw ? w[2][lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) {
            mr = max_nan(mr, __shfl_down_sync(0xffffffffu, mr, off));
            mx = max_nan(mx, __shfl_down_sync(0xffffffffu, mx, off));
            mb = max_nan(mb, __shfl_down_sync(0xffffffffu, mb, off));
        }
        if (lane == 0) { out[3 * c] = mr; out[3 * c + 1] = mx; out[3 * c + 2] = mb; }
    }
}

// Per-column error measures of a solution X of A X = B with residual R = B - A X:
// out[5c..5c+4] = max|R|, max|X|, max|B|, sum |R|^2, sum |B|^2 (one CTA per column;
// NaN propagates through every entry).
__global__ void k_col_errs5(int m, const double2 *R, int64_t ldr, const double2 *X, int64_t ldx, const double2 *B,
                            int64_t ldb, double *out) {
    const int c = blockIdx.x;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
        const double2 a = R[(int64_t)c * ldr + r];
        const double2 x = X[(int64_t)c * ldx + r];
        const double2 b = B[(int64_t)c * ldb + r];
        v[0] = max_nan(v[0], hypot(a.x, a.y));
        v[1] = max_nan(v[1], hypot(x.x, x.y));
        v[2] = max_nan(v[2], hypot(b.x, b.y));
        v[3] += a.x * a.x + a.y * a.y;
        v[4] += b.x * b.x + b.y * b.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int q = 0; q < 3; ++q) v[q] = max_nan(v[q], __shfl_down_sync(0xffffffffu, v[q], off));
        v[3] += __shfl_down_sync(0xffffffffu, v[3], off);
        v[4] += __shfl_down_sync(0xffffffffu, v[4], off);
    }
    __shared__ double w[5][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 5; ++q) w[q][warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < 5; ++q) v[q] = lane < nw ? w[q][lane] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
            for (int q = 0; q < 3; ++q) v[q] = max_nan(v[q], __shfl_down_sync(0xffffffffu, v[q], off));
            v[3] += __shfl_down_sync(0xffffffffu, v[3], off);
            v[4] += __shfl_down_sync(0xffffffffu, v[4], off);
        }
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 5; ++q) out[5 * c + q] = v[q];
        }
    }
}

// From k_col_errs5: berr[c] = max|R| / (anorm max|X| + max|B|) (inf where the denominator
// is 0 and the residual is not, or anything is NaN) and relres[c] = ||R||_2 / ||B||_2 (the
// bare ||R||_2 for a zero column); maxes[0..1] = their maxima (NaN-propagating).
__global__ void k_errs_finish(int ncol, const double *errs5, const double *anorm, double *berr, double *relres,
                              double *maxes) {
    double mb = 0.0, mr = 0.0;
    for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
        const double r = errs5[5 * c], x = errs5[5 * c + 1], b = errs5[5 * c + 2];
        const double r2 = sqrt(errs5[5 * c + 3]), b2 = sqrt(errs5[5 * c + 4]);
        const double den = (*anorm) * x + b;
        double e = den > 0 ? r / den : (r > 0 ? INFINITY : 0.0);
        if (!(e == e) || r != r || den != den) e = INFINITY;
        double rr = r2 / (b2 > 0 ? b2 : 1.0);
        if (!(rr == rr)) rr = INFINITY;
        if (berr) berr[c] = e;
        if (relres) relres[c] = rr;
        mb = fmax(mb, e);
        mr = fmax(mr, rr);
    }
    for (int off = 16; off > 0; off >>= 1) {
        mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, off));
        mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
    }
    __shared__ double w[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { w[0][warp] = mb; w[1][warp] = mr; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        mb = lane < nw ? w[0][lane] : 0.0;
        mr = lane < nw ? w[1][lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) {
            mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, off));
            mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
        }
        if (lane == 0) { maxes[0] = mb; maxes[1] = mr; }
    }
}

// berr[c] = r / (anorm x + b); relres[c] = r / b (reference RefinedLU measure).
__global__ void k_berr_finish(int ncol, const double *absmax3, const double *anorm, double *berr, double *relres,
                              double *maxes) {
    double mb = 0.0, mr = 0.0;
    for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
        const double r = absmax3[3 * c], x = absmax3[3 * c + 1], b = absmax3[3 * c + 2];
        const double den = (*anorm) * x + b;
        double e = den > 0 ? r / den : (r > 0 ? INFINITY : 0.0);
        if (!(e == e) || r != r || den != den) e = INFINITY;  // any NaN: no backward error
        double rr = r / (b > 0 ? b : 1.0);
        if (!(rr == rr)) rr = INFINITY;
        if (berr) berr[c] = e;
        if (relres) relres[c] = rr;
        mb = fmax(mb, e);
        mr = fmax(mr, rr);
    }
    for (int off = 16; off > 0; off >>= 1) {
        mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, off));
        mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
    }
    __shared__ double w[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { w[0][warp] = mb; w[1][warp] = mr; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        mb = lane < nw ? w[0][lane] : 0.0;
        mr = lane < nw ? w[1][lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) {
            mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, off));
            mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
        }
        if (lane == 0) { maxes[0] = mb; maxes[1] = mr; }
    }
}

// E[rows x cols] = 0 except E[row_off + c, c] = 1 (a shifted identity block); batched
// over blockIdx.z with stride sE.
template <typename C>
__global__ void k_set_unit(int rows, int cols, C *__restrict__ E, int64_t lde, int row_off, int64_t sE) {
    E += blockIdx.z * sE;
    const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    if (r >= rows || c >= cols) return;
    C v = czero<C>();
    if (r == row_off + c) v.x = 1;
    E[(int64_t)c * lde + r] = v;
}
