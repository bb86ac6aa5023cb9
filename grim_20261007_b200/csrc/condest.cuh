// Condition estimate of the row/column-equilibrated matrix (the reference's condition_est,
// twod/solver.py:472-577 and linalg/dense.py:157-198): B = R^-1 A C^-1 with r_i = max_j |a_ij|
// and c_j = max_i |a_ij| / r_i (zero maxima replaced by 1), cond_1(B) = ||B||_1 est(||B^-1||_1).
// The estimate of ||B^-1||_1 follows Hager's method with Higham's refinements (the iteration of
// LAPACK's zlacn2: at most five adjoint solves, then the alternating-sign test vector); the
// host drives it, these kernels do its vector steps on the device.
#pragma once
#include "common.cuh"

// r_i = max_j |a_ij| (bits of the non-negative double; row maxima combined by atomicMax).
// grid (ceil(n / 256), column chunks): each thread one row over a chunk of columns.
__global__ void k_cond_rowmax(int n, const double2 *__restrict__ A, int64_t lda, int cols_per_chunk,
                              unsigned long long *__restrict__ rmax) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c0 = blockIdx.y * cols_per_chunk, c1 = min(n, c0 + cols_per_chunk);
    double m = 0.0;
    for (int c = c0; c < c1; ++c) {
        const double2 a = A[(int64_t)c * lda + i];
        m = fmax(m, hypot(a.x, a.y));
    }
    atomicMax(&rmax[i], (unsigned long long)__double_as_longlong(m));
}

// Per column (one CTA each): c_j = max_i |a_ij| / r_i (1 when zero) and the column sum of
// the equilibrated |b_ij| = |a_ij| / (r_i c_j); r from k_cond_rowmax (1 where zero).
__global__ void __launch_bounds__(256) k_cond_cols(int n, const double2 *__restrict__ A, int64_t lda,
                                                   const unsigned long long *__restrict__ rmax,
                                                   double *__restrict__ cscale, double *__restrict__ colsum) {
    __shared__ double red[256];
    const int j = blockIdx.x;
    const double2 *a = A + (int64_t)j * lda;
    double m = 0.0, s = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) {
        double r = __longlong_as_double((long long)rmax[i]);
        r = r > 0.0 ? r : 1.0;
        const double v = hypot(a[i].x, a[i].y) / r;
        m = fmax(m, v);
        s += v;
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    const double c = red[0] > 0.0 ? red[0] : 1.0;
    __syncthreads();
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        cscale[j] = c;
        colsum[j] = red[0] / c;
    }
}

// out = max of v[0..n) (one CTA of 1024 threads; NaN propagates).
__global__ void __launch_bounds__(1024) k_cond_max(int n, const double *__restrict__ v, double *__restrict__ out) {
    __shared__ double red[1024];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) m = (v[i] > m || v[i] != v[i]) ? v[i] : m;
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            const double b = red[threadIdx.x + o];
            if (b > red[threadIdx.x] || b != b) red[threadIdx.x] = b;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// Test vectors: mode 0 x_i = 1/n; 1 x = e_j; 2 x_i = (-1)^i (1 + i / (n - 1)) (zlacn2's
// alternating-sign vector, 0-based i).
__global__ void k_cond_fill(int n, double2 *__restrict__ x, int mode, int j) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v;
    if (mode == 0) v = 1.0 / n;
    else if (mode == 1) v = i == j ? 1.0 : 0.0;
    else v = (i & 1 ? -1.0 : 1.0) * (1.0 + (n > 1 ? (double)i / (n - 1) : 0.0));
    x[i] = make_double2(v, 0.0);
}

// v_i *= s_i (rmax as double bits when bits != 0, zero maxima read as 1).
__global__ void k_cond_scale(int n, double2 *__restrict__ v, const double *__restrict__ s,
                             const unsigned long long *__restrict__ sbits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double f;
    if (s) f = s[i];
    else {
        f = __longlong_as_double((long long)sbits[i]);
        f = f > 0.0 ? f : 1.0;
    }
    v[i].x *= f;
    v[i].y *= f;
}

// One CTA of 1024 threads: out[0] = ||y||_1; with x non-null, x = sign(y) (y_i / |y_i|, 1
// where y_i = 0).
__global__ void __launch_bounds__(1024) k_cond_norm_sign(int n, const double2 *__restrict__ y,
                                                         double2 *__restrict__ x, double *__restrict__ out) {
    __shared__ double red[1024];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) {
        const double a = hypot(y[i].x, y[i].y);
        s += a;
        if (x) x[i] = a > 0.0 ? make_double2(y[i].x / a, y[i].y / a) : make_double2(1.0, 0.0);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

// One CTA of 1024 threads: the first index of the largest |z_i| (out_i[0]), that magnitude
// (out_d[0]) and |z_jlast| (out_d[1]).
__global__ void __launch_bounds__(1024) k_cond_argmax(int n, const double2 *__restrict__ z, int jlast,
                                                      int *__restrict__ out_i, double *__restrict__ out_d) {
    __shared__ double rv[1024];
    __shared__ int ri[1024];
    double bv = -1.0;
    int bi = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += 1024) {
        const double a = hypot(z[i].x, z[i].y);
        if (a > bv) {  // increasing i per thread: the first of equal values stays
            bv = a;
            bi = i;
        }
    }
    rv[threadIdx.x] = bv;
    ri[threadIdx.x] = bi;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            const double v = rv[threadIdx.x + o];
            const int k = ri[threadIdx.x + o];
            if (v > rv[threadIdx.x] || (v == rv[threadIdx.x] && k < ri[threadIdx.x])) {
                rv[threadIdx.x] = v;
                ri[threadIdx.x] = k;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out_i[0] = ri[0] == 0x7fffffff ? 0 : ri[0];
        out_d[0] = rv[0];
        out_d[1] = (jlast >= 0 && jlast < n) ? hypot(z[jlast].x, z[jlast].y) : -1.0;
    }
}

// B = conj(A)^T (tiled through shared memory).
__global__ void k_conj_transpose(int n, const double2 *__restrict__ A, int64_t lda, double2 *__restrict__ B,
                                 int64_t ldb) {
    __shared__ double2 t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = bx + threadIdx.x, c = by + k;
        if (r < n && c < n) t[k][threadIdx.x] = A[(int64_t)c * lda + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = by + threadIdx.x, c = bx + k;  // B[r][c] = conj(A[c][r])
        if (r < n && c < n) {
            const double2 v = t[threadIdx.x][k];
            B[(int64_t)c * ldb + r] = make_double2(v.x, -v.y);
        }
    }
}
