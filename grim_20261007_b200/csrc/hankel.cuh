// In-kernel Bessel / Hankel evaluation for the 2-D Green's function
//   S(R)     = (j/4) H0^(2)(kR) = (Y0 + j J0)/4
//   dS/dn(R) = -(k/4) (Y1 + j J1)(kR) (Rhat . n)
//
// FP64 path: CUDA's double-precision j0/y0/j1/y1 are called directly.
// FP32 path (written here from DLMF):
//   * x < GRIM_SMALL_KR: power series in FP64 (DLMF 10.2.2 for J, 10.8.1-2 for Y),
//     term-wise, summed until the term falls below 1e-17 of the running size;
//   * x >= GRIM_SMALL_KR: Hankel asymptotic expansion (DLMF 10.17.3-4)
//       H^(2)_nu(x) ~ sqrt(2/(pi x)) e^{-j w} sum_k (-j)^k a_k(nu) / x^k,
//       w = x - nu pi/2 - pi/4,
//       a_0 = 1, a_k(nu) = a_{k-1}(nu) (4 nu^2 - (2k-1)^2) / (8k),
//     in FP32 with GRIM_ASYM_TERMS terms (|a_8/12^8| < 2e-8 for nu = 0, 1); the phase
//     w is formed and reduced modulo 2 pi in FP64 before the FP32 sincos.
#pragma once
#include <cuda_runtime.h>

#define GRIM_SMALL_KR 12.0
#define GRIM_ASYM_TERMS 9
#define GRIM_EULER_GAMMA 0.57721566490153286
#define GRIM_PI 3.14159265358979323846
#define GRIM_TWO_PI 6.28318530717958647692

// a_k(0) and a_k(1), k = 0..GRIM_ASYM_TERMS-1 (uploaded from the host recurrence).
__constant__ float c_asym_a0[GRIM_ASYM_TERMS];
__constant__ float c_asym_a1[GRIM_ASYM_TERMS];

// ---------------------------------------------------------------- FP64 (library calls)
__device__ __forceinline__ void bessel01_fp64(double x, double &j0v, double &y0v) {
    j0v = j0(x);
    y0v = y0(x);
}
__device__ __forceinline__ void bessel11_fp64(double x, double &j1v, double &y1v) {
    j1v = j1(x);
    y1v = y1(x);
}

// ---------------------------------------------------------------- FP64 small-argument series
// J0 and Y0 for 0 < x < GRIM_SMALL_KR.
__device__ __forceinline__ void series_j0y0(double x, double &j0v, double &y0v) {
    const double q = 0.25 * x * x;  // x^2/4
    double term = 1.0;              // (-q)^s / (s!)^2
    double sj = 1.0, sy = 0.0, harm = 0.0;
    for (int s = 1; s < 80; ++s) {
        term *= -q / ((double)s * (double)s);
        harm += 1.0 / (double)s;
        sj += term;
        sy += harm * term;
        if (fabs(term) * (1.0 + harm) < 1e-17 * (fabs(sj) + 1e-300) && s > 2) break;
    }
    j0v = sj;
    y0v = (2.0 / GRIM_PI) * ((log(0.5 * x) + GRIM_EULER_GAMMA) * sj - sy);
}

// J1 and Y1 for 0 < x < GRIM_SMALL_KR.
//   J1 = (x/2) sum (-q)^s / (s!(s+1)!)
//   Y1 = -2/(pi x) + (2/pi)(ln(x/2)+gamma) J1 - (x/(2 pi)) sum (H_s + H_{s+1}) (-q)^s/(s!(s+1)!)
__device__ __forceinline__ void series_j1y1(double x, double &j1v, double &y1v) {
    const double q = 0.25 * x * x;
    double term = 1.0;  // (-q)^s / (s!(s+1)!)
    double sj = 1.0;
    double hs = 0.0, hs1 = 1.0;  // H_s, H_{s+1}
    double sy = hs + hs1;        // s = 0 term: (H_0 + H_1) * 1
    for (int s = 1; s < 80; ++s) {
        term *= -q / ((double)s * (double)(s + 1));
        hs += 1.0 / (double)s;
        hs1 += 1.0 / (double)(s + 1);
        sj += term;
        sy += (hs + hs1) * term;
        if (fabs(term) * (1.0 + hs1) < 1e-17 * (fabs(sj) + 1e-300) && s > 2) break;
    }
    const double half = 0.5 * x;
    j1v = half * sj;
    y1v = -2.0 / (GRIM_PI * x) + (2.0 / GRIM_PI) * (log(half) + GRIM_EULER_GAMMA) * j1v - (x / (2.0 * GRIM_PI)) * sy;
}

// ---------------------------------------------------------------- FP32 asymptotic
// Returns (J_nu, Y_nu)(x) for nu in {0, 1}, x >= GRIM_SMALL_KR, FP32 arithmetic
// except the phase reduction.
template <int NU>
__device__ __forceinline__ void asym_jy_fp32(double x, float &jv, float &yv) {
    const float xf = (float)x;
    const float inv = 1.0f / xf;
    const float inv2 = inv * inv;
    const float *a = NU == 0 ? c_asym_a0 : c_asym_a1;
    // P = sum_m (-1)^m a_{2m} x^{-2m},  Q = sum_m (-1)^m a_{2m+1} x^{-2m-1}
    float pp = 0.0f, qq = 0.0f, pw = 1.0f;
#pragma unroll
    for (int m = 0; 2 * m < GRIM_ASYM_TERMS; ++m) {
        const float sgn = (m & 1) ? -1.0f : 1.0f;
        pp += sgn * a[2 * m] * pw;
        if (2 * m + 1 < GRIM_ASYM_TERMS) qq += sgn * a[2 * m + 1] * pw * inv;
        pw *= inv2;
    }
    // phase w = x - nu pi/2 - pi/4, reduced in FP64
    double w = x - (0.5 * NU + 0.25) * GRIM_PI;
    w = w - GRIM_TWO_PI * rint(w / GRIM_TWO_PI);
    float sw, cw;
    sincosf((float)w, &sw, &cw);
    const float amp = sqrtf(2.0f / ((float)GRIM_PI * xf));
    jv = amp * (pp * cw - qq * sw);
    yv = amp * (pp * sw + qq * cw);
}
