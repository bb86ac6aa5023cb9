// 2-D pulse-basis, point-matched system-matrix fill, plane-wave excitation and
// matched monostatic far-field projection.
//
// Entry (m, n) of the TM EFIE / TE MFIE matrix (m = observation panel midpoint c_m,
// n = source panel):
//   TM: Z_mn = sum_q w_q h_n S(|c_m - y_nq|),          S = (j/4) H0^(2)(kR)
//   TE: Z_mn = sum_q w_q h_n dS/dn_m(c_m, y_nq),       dS/dn = -(k/4)(Y1 + jJ1)(kR) Rhat.n_m
//   y_nq = c_n + x_q h_n t_n with Gauss-Legendre (x_q, w_q) of order 12 / 6 / 4 when
//   delta = dist(c_m, panel n)/h_n is < 2 / < 6 / otherwise.
//   Diagonal: TM int_{-h}^{h} S(|t|) dt by the integrated series of J0, Y0 (FP64);
//             TE 1/2 + diag_extra[m].
// Reference: twod/operators.py:1577-1624 (Green's function and its normal derivative),
// twod/operators.py:418-501 (log-singular self term by series), operators.py:2087-2607
// (assembly loop); the reference integrates linear Galerkin elements, this path
// collocates pulse bases.
//
// Layout: Z column-major, the 32 lanes of a warp own 32 consecutive rows of one
// column, so every store is a coalesced 512 B (complex128) or 256 B (complex64) line.
// Source-panel geometry of the CTA's 32 columns is staged in shared memory.
#pragma once
#include "common.cuh"
#include "hankel.cuh"

// Gauss-Legendre nodes/weights: order q stored at offset q*(q-1)/2.
__constant__ double c_gl_x[GRIM_MAX_GAUSS * (GRIM_MAX_GAUSS + 1) / 2];
__constant__ double c_gl_w[GRIM_MAX_GAUSS * (GRIM_MAX_GAUSS + 1) / 2];

#define FILL_ROWS 32
#define FILL_COLS 32
#define FILL_WARPS 8

struct PanelGeom {
    double cx, cy, tx, ty, h, nx, ny;
};

__device__ __forceinline__ PanelGeom load_geom(const double *g, int i) {
    const double *p = g + 7 * (int64_t)i;
    PanelGeom r;
    r.cx = p[0]; r.cy = p[1]; r.tx = p[2]; r.ty = p[3]; r.h = p[4]; r.nx = p[5]; r.ny = p[6];
    return r;
}

__device__ __forceinline__ int quad_order_for(double ox, double oy, const PanelGeom &s) {
    const double dx = ox - s.cx, dy = oy - s.cy;
    double along = dx * s.tx + dy * s.ty;
    along = fmin(fmax(along, -s.h), s.h);
    const double ex = dx - along * s.tx, ey = dy - along * s.ty;
    const double delta = hypot(ex, ey) / s.h;
    return delta < 2.0 ? 12 : (delta < 6.0 ? 6 : 4);
}

// int_{-h}^{h} (j/4) H0^(2)(k|t|) dt = (j/(2k)) int_0^{kh} (J0 - j Y0) du
__device__ double2 tm_self_term(double k, double h) {
    const double x = k * h;
    const double lx = log(0.5 * x);
    double ij = 0.0, iy = 0.0, c = 1.0, harm = 0.0, p = x;
    for (int s = 0; s < 200; ++s) {
        if (s > 0) {
            c *= -1.0 / (4.0 * (double)s * (double)s);
            harm += 1.0 / (double)s;
            p *= x * x;
        }
        const double term = c * p / (double)(2 * s + 1);
        ij += term;
        iy += term * (lx + GRIM_EULER_GAMMA - 1.0 / (double)(2 * s + 1) - harm);
        if (s > 4 && fabs(term) * (1.0 + fabs(lx) + harm) < 1e-18 * fmax(1.0, fabs(ij))) break;
    }
    iy *= 2.0 / GRIM_PI;
    // (j/(2k)) * (ij - j iy) = (iy + j ij) / (2k)
    return make_double2(iy / (2.0 * k), ij / (2.0 * k));
}

// One off-diagonal entry, FP64.
template <int POL>
__device__ __forceinline__ double2 entry_fp64(double k, double ox, double oy, double onx, double ony,
                                              const PanelGeom &s) {
    const int q = quad_order_for(ox, oy, s);
    const int off = q * (q - 1) / 2;
    double re = 0.0, im = 0.0;
    for (int i = 0; i < q; ++i) {
        const double xq = c_gl_x[off + i], wq = c_gl_w[off + i] * s.h;
        const double dx = ox - (s.cx + xq * s.h * s.tx);
        const double dy = oy - (s.cy + xq * s.h * s.ty);
        const double r = hypot(dx, dy);
        const double kr = k * r;
        if (POL == GRIM_POL_TM) {
            double jv, yv;
            bessel01_fp64(kr, jv, yv);
            re += wq * 0.25 * yv;
            im += wq * 0.25 * jv;
        } else {
            double jv, yv;
            bessel11_fp64(kr, jv, yv);
            const double rdn = (dx * onx + dy * ony) / r;
            const double f = -0.25 * k * rdn * wq;
            re += f * yv;
            im += f * jv;
        }
    }
    return make_double2(re, im);
}

// One off-diagonal entry, complex64 output: FP64 series below GRIM_SMALL_KR,
// FP32 asymptotic above; geometry differences and phases in FP64.
template <int POL>
__device__ __forceinline__ float2 entry_fp32(double k, double ox, double oy, double onx, double ony,
                                             const PanelGeom &s) {
    const int q = quad_order_for(ox, oy, s);
    const int off = q * (q - 1) / 2;
    float re = 0.f, im = 0.f;
    double red = 0.0, imd = 0.0;
    for (int i = 0; i < q; ++i) {
        const double xq = c_gl_x[off + i], wq = c_gl_w[off + i] * s.h;
        const double dx = ox - (s.cx + xq * s.h * s.tx);
        const double dy = oy - (s.cy + xq * s.h * s.ty);
        const double r = sqrt(dx * dx + dy * dy);
        const double kr = k * r;
        if (kr < GRIM_SMALL_KR) {
            double jv, yv;
            if (POL == GRIM_POL_TM) {
                series_j0y0(kr, jv, yv);
                red += wq * 0.25 * yv;
                imd += wq * 0.25 * jv;
            } else {
                series_j1y1(kr, jv, yv);
                const double f = -0.25 * k * wq * (dx * onx + dy * ony) / r;
                red += f * yv;
                imd += f * jv;
            }
        } else {
            float jv, yv;
            if (POL == GRIM_POL_TM) {
                asym_jy_fp32<0>(kr, jv, yv);
                const float f = (float)(wq * 0.25);
                re = fmaf(f, yv, re);
                im = fmaf(f, jv, im);
            } else {
                asym_jy_fp32<1>(kr, jv, yv);
                const float f = (float)(-0.25 * k * wq * ((dx * onx + dy * ony) / r));
                re = fmaf(f, yv, re);
                im = fmaf(f, jv, im);
            }
        }
    }
    return make_float2((float)(red + (double)re), (float)(imd + (double)im));
}

template <int POL, typename C>
__global__ void __launch_bounds__(FILL_ROWS * FILL_WARPS)
k_fill2d(int n, const double *__restrict__ geom, const double *__restrict__ diag_extra, double k,
         C *__restrict__ Z, int64_t ldz) {
    __shared__ PanelGeom sg[FILL_COLS];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int row0 = blockIdx.x * FILL_ROWS;
    const int col0 = blockIdx.y * FILL_COLS;
    if (threadIdx.x < FILL_COLS && col0 + (int)threadIdx.x < n) sg[threadIdx.x] = load_geom(geom, col0 + threadIdx.x);
    __syncthreads();
    const int m = row0 + lane;
    if (m >= n) return;
    const PanelGeom o = load_geom(geom, m);
    for (int cc = warp; cc < FILL_COLS; cc += FILL_WARPS) {
        const int col = col0 + cc;
        if (col >= n) break;
        C val;
        if (col == m) {
            double2 d;
            if (POL == GRIM_POL_TM) d = tm_self_term(k, o.h);
            else d = make_double2(0.5 + (diag_extra ? diag_extra[m] : 0.0), 0.0);
            val = conv<C>(d);
        } else {
            if constexpr (sizeof(C) == sizeof(double2)) {
                val = conv<C>(entry_fp64<POL>(k, o.cx, o.cy, o.nx, o.ny, sg[cc]));
            } else {
                float2 v = entry_fp32<POL>(k, o.cx, o.cy, o.nx, o.ny, sg[cc]);
                val = *reinterpret_cast<C *>(&v);
            }
        }
        Z[(int64_t)col * ldz + m] = val;
    }
}

// Plane-wave excitation, one thread per (row, angle).
template <int POL, typename C>
__global__ void k_rhs2d(int n, const double *__restrict__ geom, int nang, const double *__restrict__ ang_deg,
                        double k, C *__restrict__ B, int64_t ldb) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    if (m >= n || a >= nang) return;
    const PanelGeom o = load_geom(geom, m);
    double sphi, cphi;
    sincospi(ang_deg[a] / 180.0, &sphi, &cphi);
    const double ph = k * (cphi * o.cx + sphi * o.cy);
    double s, c;
    sincos(ph, &s, &c);
    double2 v;
    if (POL == GRIM_POL_TM) {
        v = make_double2(-c, -s);
    } else {
        const double dn = k * (cphi * o.nx + sphi * o.ny);  // -j k dn e^{j ph}
        v = make_double2(dn * s, -dn * c);
    }
    B[(int64_t)a * ldb + m] = conv<C>(v);
}

// Matched monostatic far field: amp[a] = sum_n X[n,a] w_n(a); one CTA per angle,
// fixed-order tree reduction (bitwise reproducible for a given n).
template <typename C>
__global__ void k_farfield2d(int n, const double *__restrict__ geom, int nang, const double *__restrict__ ang_deg,
                             double k, const C *__restrict__ X, int64_t ldx, double2 *__restrict__ amp) {
    const int a = blockIdx.x;
    if (a >= nang) return;
    double sphi, cphi;
    sincospi(ang_deg[a] / 180.0, &sphi, &cphi);
    double re = 0.0, im = 0.0;
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        const PanelGeom o = load_geom(geom, m);
        const double arg = k * (cphi * o.tx + sphi * o.ty) * o.h;
        const double sinc = fabs(arg) < 1e-8 ? 1.0 - arg * arg / 6.0 : sin(arg) / arg;
        double s, c;
        sincos(k * (cphi * o.cx + sphi * o.cy), &s, &c);
        const double wr = 2.0 * o.h * sinc * c, wi = 2.0 * o.h * sinc * s;
        const double2 x = to_c64(X[(int64_t)a * ldx + m]);
        re += x.x * wr - x.y * wi;
        im += x.x * wi + x.y * wr;
    }
    __shared__ double sr[32], si[32];
    for (int off = 16; off > 0; off >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, off);
        im += __shfl_down_sync(0xffffffffu, im, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sr[warp] = re; si[warp] = im; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        re = lane < nw ? sr[lane] : 0.0;
        im = lane < nw ? si[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) {
            re += __shfl_down_sync(0xffffffffu, re, off);
            im += __shfl_down_sync(0xffffffffu, im, off);
        }
        if (lane == 0) amp[a] = make_double2(re, im);
    }
}
