// Far-field Galerkin element-pair blocks of the reference's linear-Galerkin 2-D fill
// (twod/assembly/native/far.c:100-207 ghost_far_block, the native form of the far pass of
// twod/operators.py:2087-2607 _assemble_multi), on the GPU.
//
// For every pair (i, j) of observation element i and source element j marked in `far`:
//   S[a b]  = sum_qi wo_qi phi_a(qi) sum_qj w_qj phi_b(qj) G(r)
//   K[a b]  = ... dG(r) (r^ . n)         (n = observation normal if obs_normal_deriv,
//   Kt[a b] = ... the mirrored kernel     else the source normal; signs as the reference)
// with G = (j/4) H0^(2)(kr) and dG = (j/4) k H1^(2)(kr) read from the caller's
// piecewise-polynomial kernel table (normalized power coefficients, Horner in the interval
// coordinate) and, beyond the table, the 8-term large-argument Hankel expansion.
//
// One thread per pair.  The arithmetic is the reference's, operation for operation and in
// the same order, with every product, sum, quotient and square root rounded on its own
// (__dmul_rn / __dadd_rn / __ddiv_rn / __dsqrt_rn: no fused multiply-add), so a pair whose
// distances all fall inside the table receives bitwise the reference's sums.  Beyond the
// table the exponential and trigonometric functions are CUDA's (agreement to a few ulp).
// The accumulators are read once, summed in registers in the reference's order
// (acc = acc + term per observation point) and written once.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define FAR_EPS 1e-12
#define FAR_MAX_WIDTH 8
#define FAR_DEGREE 12  // the reference tables' polynomial degree (twod/assembly/kernels.py:338)
#define FAR_SMEM_BOUNDS 4097  // tables up to 4096 intervals keep their bounds in shared memory

struct FarTable {
    int intervals, degree;
    const double *bounds, *coeff;
    double k_re, k_im;
    int coeff16;  // coeff is 16-byte aligned: (re, im) pairs are read as one 16-byte load
};

__device__ __forceinline__ double far_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double far_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double far_sub(double a, double b) { return __dsub_rn(a, b); }

// Principal complex square root.
__device__ __forceinline__ void far_csqrt(double a, double b, double *re, double *im) {
    const double m = hypot(a, b);
    if (m == 0.0) {
        *re = 0.0;
        *im = b;
        return;
    }
    if (a >= 0.0) {
        const double t = sqrt(0.5 * (m + a));
        *re = t;
        *im = b / (2.0 * t);
    } else {
        const double t = sqrt(0.5 * (m - a));
        *re = fabs(b) / (2.0 * t);
        *im = copysign(t, b);
    }
}

// (j/4) H0^(2)(kr) and (j/4) k H1^(2)(kr) for |kr| >= 128 (eight terms of the
// large-argument expansion).
__device__ void far_asymptotic(const FarTable &t, double r, double *out) {
    const double pi = 3.14159265358979323846;
    const double zr = t.k_re * r, zi = t.k_im * r;
    // root = sqrt(2 / (pi z))
    const double den = pi * (zr * zr + zi * zi);
    double rr, ri;
    far_csqrt(2.0 * zr / den, -2.0 * zi / den, &rr, &ri);
    // factor = -j / z = -j conj(z) / |z|^2
    const double zz = zr * zr + zi * zi;
    const double fr = -zi / zz, fi = -zr / zz;
    for (int nu = 0; nu < 2; ++nu) {
        const double mu = 4.0 * nu * nu;
        double tr = 1.0, ti = 0.0, sr = 1.0, si = 0.0;
        for (int m = 1; m < 8; ++m) {
            const double odd = 2.0 * m - 1.0;
            const double c = (mu - odd * odd) / (8.0 * m);
            const double ar = c * fr, ai = c * fi;
            const double nr = tr * ar - ti * ai, ni = tr * ai + ti * ar;
            tr = nr;
            ti = ni;
            sr += tr;
            si += ti;
        }
        // phase = exp(-j (z - nu pi/2 - pi/4))
        const double ur = zr - nu * pi / 2.0 - pi / 4.0, ui = zi;
        double sn, cs;
        sincos(ur, &sn, &cs);
        const double e = exp(ui);
        const double pr = e * cs, pi_ = -e * sn;
        // value = 0.25 j root phase sum
        const double a1r = rr * pr - ri * pi_, a1i = rr * pi_ + ri * pr;
        const double a2r = a1r * sr - a1i * si, a2i = a1r * si + a1i * sr;
        double vr = -0.25 * a2i, vi = 0.25 * a2r;
        if (nu == 1) {
            const double wr = vr * t.k_re - vi * t.k_im, wi = vr * t.k_im + vi * t.k_re;
            vr = wr;
            vi = wi;
        }
        out[2 * nu] = vr;
        out[2 * nu + 1] = vi;
    }
}

// Kernel values at distance r: false below the table (the caller's fallback case).
__device__ __forceinline__ bool far_kernel(const FarTable &t, double r, double *out) {
    const double *bounds = t.bounds;
    if (!(r >= bounds[0])) return false;
    if (r > bounds[t.intervals]) {
        far_asymptotic(t, r, out);
        return true;
    }
    int lo = 0, hi = t.intervals;
    while (lo + 1 < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (r < bounds[mid]) hi = mid;
        else lo = mid;
    }
    const double b0 = bounds[lo], b1 = bounds[lo + 1];
    const double x = __ddiv_rn(far_sub(r, b0), far_sub(b1, b0));
    const double *base = t.coeff + (int64_t)lo * (t.degree + 1) * 4;
    if (t.degree == FAR_DEGREE && t.coeff16) {
        // the usual degree: both channels' Horner chains interleaved, (re, im) pairs read
        // as 16-byte loads that the unrolled loop can issue ahead of their use
        const double2 *b2 = reinterpret_cast<const double2 *>(base);
        double2 g = __ldg(b2 + 2 * FAR_DEGREE), d = __ldg(b2 + 2 * FAR_DEGREE + 1);
#pragma unroll
        for (int j = FAR_DEGREE - 1; j >= 0; --j) {
            const double2 cg = __ldg(b2 + 2 * j), cd = __ldg(b2 + 2 * j + 1);
            g.x = far_add(far_mul(g.x, x), cg.x);
            g.y = far_add(far_mul(g.y, x), cg.y);
            d.x = far_add(far_mul(d.x, x), cd.x);
            d.y = far_add(far_mul(d.y, x), cd.y);
        }
        out[0] = g.x;
        out[1] = g.y;
        out[2] = d.x;
        out[3] = d.y;
        return true;
    }
    for (int c = 0; c < 2; ++c) {
        const int off = 2 * c;
        double re = __ldg(base + 4 * t.degree + off), im = __ldg(base + 4 * t.degree + off + 1);
        for (int j = t.degree - 1; j >= 0; --j) {
            re = far_add(far_mul(re, x), __ldg(base + 4 * j + off));
            im = far_add(far_mul(im, x), __ldg(base + 4 * j + off + 1));
        }
        out[2 * c] = re;
        out[2 * c + 1] = im;
    }
    return true;
}

__device__ __forceinline__ void far_first_or_add(double *acc, bool first, double re, double im, double c) {
    if (first) {
        acc[0] = far_mul(re, c);
        acc[1] = far_mul(im, c);
    } else {
        acc[0] = far_add(acc[0], far_mul(re, c));
        acc[1] = far_add(acc[1], far_mul(im, c));
    }
}

// W > 0: compile-time width (accumulators in registers); W = 0: runtime width <= 8.
// MINB: CTAs per SM the register allocation must allow.
template <int W, int MINB>
__global__ void __launch_bounds__(128, MINB)
k_far_block(int64_t mb, int64_t nb, int q, int width_rt, const double *__restrict__ obs_pts,
            const double *__restrict__ src_pts, const double *__restrict__ qw, const double *__restrict__ phi,
            const double *__restrict__ obs_norm, const double *__restrict__ src_norm, const uint8_t *__restrict__ far,
            int obs_normal_deriv, int want_s, int want_k, int mirrored, FarTable table, double *acc_s, double *acc_k,
            double *acc_kt, int *status) {
    constexpr int MW = W > 0 ? W : FAR_MAX_WIDTH;
    const int width = W > 0 ? W : width_rt;
    const int64_t plane = mb * nb;
    const int64_t pair = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // the table's interval bounds in shared memory (the binary search reads them most)
    extern __shared__ double s_bounds[];
    if (table.intervals + 1 <= FAR_SMEM_BOUNDS) {
        for (int e = threadIdx.x; e <= table.intervals; e += blockDim.x) s_bounds[e] = table.bounds[e];
        __syncthreads();
        table.bounds = s_bounds;
    }
    if (pair >= plane || !far[pair]) return;
    const int64_t i = pair / nb, j = pair % nb;
    const bool with_kt = want_k && mirrored;
    const double *on = obs_norm + 2 * i, *sn = src_norm + 2 * j;
    const double *n_ij = obs_normal_deriv ? on : sn;
    const double *n_ji = obs_normal_deriv ? sn : on;
    const double nij0 = n_ij[0], nij1 = n_ij[1], nji0 = n_ji[0], nji1 = n_ji[1];
    double as[MW * MW][2], ak[MW * MW][2], akt[MW * MW][2];
    for (int ab = 0; ab < width * width; ++ab) {
        const int64_t at = ((int64_t)ab * plane + pair) * 2;
        if (want_s) { as[ab][0] = acc_s[at]; as[ab][1] = acc_s[at + 1]; }
        if (want_k) { ak[ab][0] = acc_k[at]; ak[ab][1] = acc_k[at + 1]; }
        if (with_kt) { akt[ab][0] = acc_kt[at]; akt[ab][1] = acc_kt[at + 1]; }
    }
    for (int qi = 0; qi < q; ++qi) {
        double ps[MW][2], pk[MW][2], pkt[MW][2];
        const double ox = obs_pts[(i * q + qi) * 2], oy = obs_pts[(i * q + qi) * 2 + 1];
        for (int qj = 0; qj < q; ++qj) {
            const double dx = far_sub(ox, src_pts[(j * q + qj) * 2]);
            const double dy = far_sub(oy, src_pts[(j * q + qj) * 2 + 1]);
            double dist = __dsqrt_rn(far_add(far_mul(dx, dx), far_mul(dy, dy)));
            if (!(dist >= FAR_EPS)) dist = FAR_EPS;
            double value[4];
            if (!far_kernel(table, dist, value)) {
                atomicOr(status, 2);
                return;
            }
            const double w = qw[qj];
            const double *phi_s = phi + qj * width;
            const bool first = qj == 0;
            double dk_re = 0.0, dk_im = 0.0;
            if (want_k) {
                const double proj = __ddiv_rn(far_add(far_mul(dx, nij0), far_mul(dy, nij1)), dist);
                dk_re = far_mul(value[2], proj);
                dk_im = far_mul(value[3], proj);
                if (obs_normal_deriv) {
                    dk_re = -dk_re;
                    dk_im = -dk_im;
                }
            }
#pragma unroll
            for (int b = 0; b < MW; ++b) {
                if (b >= width) break;
                const double c = far_mul(w, phi_s[b]);
                if (want_s) far_first_or_add(ps[b], first, value[0], value[1], c);
                if (want_k) far_first_or_add(pk[b], first, dk_re, dk_im, c);
            }
            if (with_kt) {
                const double proj = __ddiv_rn(far_add(far_mul(dx, nji0), far_mul(dy, nji1)), dist);
                double re = far_mul(value[2], proj), im = far_mul(value[3], proj);
                if (!obs_normal_deriv) {
                    re = -re;
                    im = -im;
                }
#pragma unroll
                for (int a = 0; a < MW; ++a) {
                    if (a >= width) break;
                    far_first_or_add(pkt[a], first, re, im, far_mul(w, phi_s[a]));
                }
            }
        }
        const double wo = qw[qi];
        const double *phi_o = phi + qi * width;
#pragma unroll
        for (int a = 0; a < MW; ++a) {
            if (a >= width) break;
            const double c = far_mul(wo, phi_o[a]);
#pragma unroll
            for (int b = 0; b < MW; ++b) {
                if (b >= width) break;
                const int ab = width * a + b;
                if (want_s) {
                    as[ab][0] = far_add(as[ab][0], far_mul(ps[b][0], c));
                    as[ab][1] = far_add(as[ab][1], far_mul(ps[b][1], c));
                }
                if (want_k) {
                    ak[ab][0] = far_add(ak[ab][0], far_mul(pk[b][0], c));
                    ak[ab][1] = far_add(ak[ab][1], far_mul(pk[b][1], c));
                }
            }
        }
        if (with_kt) {
#pragma unroll
            for (int b = 0; b < MW; ++b) {
                if (b >= width) break;
                const double c = far_mul(wo, phi_o[b]);
#pragma unroll
                for (int a = 0; a < MW; ++a) {
                    if (a >= width) break;
                    const int ab = width * a + b;
                    akt[ab][0] = far_add(akt[ab][0], far_mul(pkt[a][0], c));
                    akt[ab][1] = far_add(akt[ab][1], far_mul(pkt[a][1], c));
                }
            }
        }
    }
    for (int ab = 0; ab < width * width; ++ab) {
        const int64_t at = ((int64_t)ab * plane + pair) * 2;
        if (want_s) { acc_s[at] = as[ab][0]; acc_s[at + 1] = as[ab][1]; }
        if (want_k) { acc_k[at] = ak[ab][0]; acc_k[at + 1] = ak[ab][1]; }
        if (with_kt) { acc_kt[at] = akt[ab][0]; acc_kt[at + 1] = akt[ab][1]; }
    }
}
