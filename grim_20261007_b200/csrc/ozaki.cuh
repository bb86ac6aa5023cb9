// Residual R = B - A X for complex A (complex64 or complex128) and complex128 X, B on the
// integer tensor cores (tcgen05 kind::i8), after the error-free slicing scheme of Ozaki
// et al. ("Error-free transformations of matrix multiplication by using fast routines of
// matrix multiplication and its applications", Numer. Algorithms 59, 2012), in its
// integer form:
//
//   every row m of A~ (the real 2n x 2n expansion [re -im; im re]) is scaled by 2^-e_m,
//   e_m one above the binary exponent of max_k max(|re|, |im|) of row m, so that
//   |a| < 1/2, and cut into S slices  a = sum_s q_s 2^-7s + rest,  q_s = rint(2^7 rest_{s-1})
//   in [-64, 64], |rest_s| <= 2^-7s / 2 (every step exact in FP64; round-to-nearest keeps
//   the remainders unbiased); every column j of X^ (rows 2k+s = re, im of X[k, j])
//   likewise with its own exponent f_j.  Then
//     (A~ X^)[r, j] ~ 2^(e_m + f_j) sum_{s + u <= S + 1} 2^-7(s+u) (Q_s P_u)[r, j]
//   where each Q_s P_u is an exact int8 x int8 -> int32 product; the pairs with the same
//   s + u share one int32 accumulator in tensor memory (S accumulators, at most S
//   products each: |sum| <= S * 2n * 64^2 < 2^31 for n < 2^31 / (2 S 64^2)).  The
//   epilogue converts the S accumulators to FP64, scales them by powers of two (exact)
//   and writes R = B - A X.  Slice remainders and the dropped terms (s + u > S + 1) are
//   below 2^-7S of 2^(e_m + f_j) per product term and of either sign.  With S = 8
//   (56 bits) the residual is as accurate as an FP64 GEMM's (measured against an
//   extended-precision product: 4e-17 vs 9e-17 of max (|A||X|); S = 7 gives 6e-15).
//
// Operand layout: the tile layout of tc_gemm.cuh with 128-byte rows of 128 int8 (K-tiles
// of 128), slice s of an operand with Rp rows and Kp columns at offset s * Rp * Kp.
//
// Kernel (one 128-row x BN-column output tile per CTA, 128 threads): X's S slice tiles of
// a K-tile sit in one of two X buffers; A's S slice tiles stream through a 4-deep ring.
// Warp 0 lane 0 issues bulk copies; warp 1 lane 0 issues, for slice tile s of A, the
// MMAs with X slices u <= S - 1 - s into accumulator s + u (4 MMAs of K 32 per pair) and
// commits to the A slot's and, after the last slice, the X buffer's "empty" barriers;
// the epilogue runs on all 4 warps.  Waits are bounded as in tc_gemm.cuh.
#pragma once
#include "tc_gemm.cuh"

#define OZ_RING 4
#define OZ_KT 128  // int8 per K-tile row (128 bytes)

// Byte offset of element (r, k) in the int8 tile layout of an operand with Rp rows.
__host__ __device__ __forceinline__ int64_t oz_tile_offset(int r, int k, int Rp) {
    return (int64_t)(k >> 7) * Rp * 128 + (int64_t)r * 128 + ((((k & 127) >> 4) ^ (r & 7)) << 4) + (k & 15);
}

template <int S, int BN>
struct OzCfg {
    static constexpr int A_BYTES = TC_BM * OZ_KT;   // one A slice tile
    static constexpr int X_BYTES = BN * OZ_KT;      // one X slice tile
    static constexpr int XBUF_BYTES = S * X_BYTES;  // all X slices of a K-tile
    static constexpr int SMEM_BYTES = 2 * XBUF_BYTES + OZ_RING * A_BYTES + 1024;
    static constexpr int TMEM_COLS = S * BN <= 256 ? 256 : 512;
    static_assert(S * BN <= 512, "accumulators exceed tensor memory");
    static_assert(BN % 16 == 0 && BN <= 256, "MMA N");
    static_assert(X_BYTES % 1024 == 0, "X tiles must keep 1024-byte atoms");
};

// max(a, b) that returns NaN when either is NaN.
__device__ __forceinline__ double oz_max_nan(double a, double b) { return (a != a) ? a : ((b != b || b > a) ? b : a); }

// Largest |component| of a complex number (NaN if a component is NaN).
template <typename T>
__device__ __forceinline__ double oz_cmax(T v) {
    return oz_max_nan(fabs((double)v.x), fabs((double)v.y));
}

// Exponent sentinel of a row or column holding Inf or NaN: its residual entries are NaN.
#define OZ_NONFINITE (-2147483647 - 1)

// Per complex row m: max over k of max(|re A|, |im A|), as the bit pattern of a
// non-negative double (monotone under unsigned compare; Inf and NaN order above every
// finite value).  rowmax zeroed by the caller; grid (ceil(n / 256), chunks), each
// thread scans a slice of one row.
template <typename TA>
__global__ void k_oz_rowmax(int n, const TA *__restrict__ A, int64_t lda, unsigned long long *rowmax) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int k0 = blockIdx.y * per, k1 = min(n, k0 + per);
    double mx = 0.0;
    for (int k = k0; k < k1; ++k) mx = oz_max_nan(mx, oz_cmax(A[(int64_t)k * lda + m]));
    if (mx != 0.0) atomicMax(rowmax + m, (unsigned long long)__double_as_longlong(mx));
}

// Per column j of X (n x nrhs): max over k of max(|re|, |im|).  One CTA (256) per column.
__global__ void k_oz_colmax(int n, const double2 *__restrict__ X, int64_t ldx, double *colmax) {
    __shared__ double red[8];
    const int j = blockIdx.x;
    double mx = 0.0;  // a NaN survives the max: a non-finite column must not look finite
    for (int k = threadIdx.x; k < n; k += blockDim.x) mx = oz_max_nan(mx, oz_cmax(X[(int64_t)j * ldx + k]));
    for (int o = 16; o > 0; o >>= 1) mx = oz_max_nan(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = oz_max_nan(mx, red[w]);
        colmax[j] = mx;
    }
}

// Exponent e with max < 2^(e-1), so scaled entries are below 1/2 (0 for a zero row or
// column, OZ_NONFINITE for Inf/NaN).
__device__ __forceinline__ int oz_exp(double mx) {
    if (!isfinite(mx)) return OZ_NONFINITE;
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    return mx > 0.0 ? e + 1 : 0;
}

// Cut 16 values (already scaled below 1/2 in magnitude) into S int8 slices in [-64, 64],
// written as one 16-byte chunk per slice at dst + s * slice_stride.
template <int S>
__device__ __forceinline__ void oz_cut16(const double (&t)[16], int8_t *dst, int64_t slice_stride) {
    double r[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) r[i] = t[i];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        uint32_t w[4];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            uint32_t word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int i = 4 * g + b;
                const double y = r[i] * 128.0;
                const double q = rint(y);
                r[i] = y - q;
                word |= ((uint32_t)(int)q & 0xffu) << (8 * b);
            }
            w[g] = word;
        }
        *reinterpret_cast<uint4 *>(dst + s * slice_stride) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Slices of A~ (rows r = 2m + t, columns 2k + c).  One thread per (complex row m, 8
// complex columns): both real rows of m, S slices each.  Grid covers Rp/2 x Kp/16.
template <typename TA, int S>
__global__ void k_oz_slice_a(int n, const TA *__restrict__ A, int64_t lda, const unsigned long long *rowmax,
                             int8_t *__restrict__ Q, int Rp, int Kp, int *row_exp) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int mrows = Rp >> 1, qn = Kp >> 4;
    if (idx >= (int64_t)mrows * qn) return;
    const int m = (int)(idx % mrows), q = (int)(idx / mrows);
    const int e = m < n ? oz_exp(__longlong_as_double((long long)rowmax[m])) : 0;
    if (q == 0 && m < n) row_exp[m] = e;
    double t0[16], t1[16];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int k = 8 * q + i;
        double re = 0.0, im = 0.0;
        if (m < n && k < n && e != OZ_NONFINITE) {
            const TA a = A[(int64_t)k * lda + m];
            re = ldexp((double)a.x, -e);
            im = ldexp((double)a.y, -e);
        }
        t0[2 * i] = re;
        t0[2 * i + 1] = -im;
        t1[2 * i] = im;
        t1[2 * i + 1] = re;
    }
    const int64_t stride = (int64_t)Rp * Kp;
    oz_cut16<S>(t0, Q + oz_tile_offset(2 * m, 16 * q, Rp), stride);
    oz_cut16<S>(t1, Q + oz_tile_offset(2 * m + 1, 16 * q, Rp), stride);
}

// Slices of X^ (rows j = right-hand sides, columns 2k + c).  One thread per (j, 8
// complex rows of X).  Grid covers Np x Kp/16.
template <int S>
__global__ void k_oz_slice_x(int n, int nrhs, const double2 *__restrict__ X, int64_t ldx, const double *colmax,
                             int8_t *__restrict__ P, int Np, int Kp, int *col_exp) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int qn = Kp >> 4;
    if (idx >= (int64_t)Np * qn) return;
    const int j = (int)(idx / qn), q = (int)(idx % qn);
    const int e = j < nrhs ? oz_exp(colmax[j]) : 0;
    if (q == 0 && j < nrhs) col_exp[j] = e;
    double t[16];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int k = 8 * q + i;
        double re = 0.0, im = 0.0;
        if (j < nrhs && k < n && e != OZ_NONFINITE) {
            const double2 x = X[(int64_t)j * ldx + k];
            re = ldexp(x.x, -e);
            im = ldexp(x.y, -e);
        }
        t[2 * i] = re;
        t[2 * i + 1] = im;
    }
    oz_cut16<S>(t, P + oz_tile_offset(j, 16 * q, Np), (int64_t)Np * Kp);
}

// One K-tile step for slice tile s of A: MMAs with X slices u <= S-1-s into accumulator s+u.
template <int S, int BN>
__device__ __forceinline__ void oz_mma_slice(uint32_t tmem, uint32_t sA, uint32_t xbuf, int s, uint32_t idesc,
                                             bool first_k) {
#pragma unroll
    for (int u = 0; u < S; ++u) {
        if (u > S - 1 - s) break;
        const uint32_t d_tmem = tmem + (uint32_t)((s + u) * BN);
        const uint32_t sX = xbuf + u * OzCfg<S, BN>::X_BYTES;
#pragma unroll
        for (int kk = 0; kk < OZ_KT / 32; ++kk) {
            const uint64_t da = umma_desc_sw128(sA + kk * 32);
            const uint64_t db = umma_desc_sw128(sX + kk * 32);
            const uint32_t acc = (first_k && s == 0 && kk == 0) ? 0u : 1u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                :
                : "r"(d_tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u)
                : "memory");
        }
    }
}

// R[r, j] = B[r, j] - 2^(e_m + f_j) sum_d 2^-7(d+2) D_d[r, j] on interleaved complex128
// (real row r = 2m + t).  grid = (Np / BN, Rp / 128).
template <int S, int BN>
__global__ void __launch_bounds__(TC_THREADS)
k_oz_gemm(int nk, const int8_t *__restrict__ Q, int Rp, const int8_t *__restrict__ P, int Np, int Kp,
          const int *__restrict__ row_exp, const int *__restrict__ col_exp, const double *__restrict__ B,
          int64_t ldb_real, double *__restrict__ R, int64_t ldr_real, int Mvalid, int Nvalid, int *err) {
    using Cfg = OzCfg<S, BN>;
    extern __shared__ __align__(1024) unsigned char smem_dyn[];
    __shared__ __align__(8) uint64_t xfull[2], xempty[2], afull[OZ_RING], aempty[OZ_RING], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;
    const uint32_t base = (smem_addr(smem_dyn) + 1023u) & ~1023u;
    const uint32_t xbase = base, abase = base + 2 * Cfg::XBUF_BYTES;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // blockIdx.x runs over the N tiles, so the CTAs resident together share A slice tiles in L2
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;
    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int i = 0; i < 2; ++i) {
            mbar_init(smem_addr(&xfull[i]), 1);
            mbar_init(smem_addr(&xempty[i]), 1);
        }
        for (int i = 0; i < OZ_RING; ++i) {
            mbar_init(smem_addr(&afull[i]), 1);
            mbar_init(smem_addr(&aempty[i]), 1);
        }
        mbar_init(smem_addr(&done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(Cfg::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    volatile int *vfail = &s_fail;
    const int64_t qstride = (int64_t)Rp * Kp, pstride = (int64_t)Np * Kp;

    if (warp == 0) {
        if (lane == 0) {
            int x_issued = 0, a_issued = 0;
            for (int kt = 0; kt < nk && !*vfail; ++kt) {
                const int xb = kt & 1;
                if (kt >= 2 && !mbar_wait(smem_addr(&xempty[xb]), ((kt >> 1) + 1) & 1)) {
                    *vfail = 1;
                    break;
                }
                const uint32_t xf = smem_addr(&xfull[xb]);
                mbar_expect_tx(xf, Cfg::XBUF_BYTES);
                for (int u = 0; u < S; ++u)
                    bulk_g2s(xbase + xb * Cfg::XBUF_BYTES + u * Cfg::X_BYTES,
                             P + u * pstride + (int64_t)kt * Np * 128 + (int64_t)n0 * 128, Cfg::X_BYTES, xf);
                x_issued = kt + 1;
                for (int s = 0; s < S; ++s) {
                    const int g = kt * S + s, slot = g % OZ_RING;
                    if (g >= OZ_RING && !mbar_wait(smem_addr(&aempty[slot]), ((g / OZ_RING) + 1) & 1)) {
                        *vfail = 1;
                        break;
                    }
                    const uint32_t af = smem_addr(&afull[slot]);
                    mbar_expect_tx(af, Cfg::A_BYTES);
                    bulk_g2s(abase + slot * Cfg::A_BYTES, Q + s * qstride + (int64_t)kt * Rp * 128 + (int64_t)m0 * 128,
                             Cfg::A_BYTES, af);
                    a_issued = g + 1;
                }
            }
            if (*vfail) {
                // let issued copies land before the CTA can exit
                for (int kt = (x_issued > 2 ? x_issued - 2 : 0); kt < x_issued; ++kt)
                    mbar_wait(smem_addr(&xfull[kt & 1]), (kt >> 1) & 1);
                for (int g = (a_issued > OZ_RING ? a_issued - OZ_RING : 0); g < a_issued; ++g)
                    mbar_wait(smem_addr(&afull[g % OZ_RING]), (g / OZ_RING) & 1);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // kind::i8: D s32 (2 << 4), A and B signed (1 << 7, 1 << 10), both K-major
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(TC_BM >> 4) << 24);
            for (int kt = 0; kt < nk && !*vfail; ++kt) {
                const int xb = kt & 1;
                if (!mbar_wait(smem_addr(&xfull[xb]), (kt >> 1) & 1)) {
                    *vfail = 1;
                    break;
                }
                for (int s = 0; s < S; ++s) {
                    const int g = kt * S + s, slot = g % OZ_RING;
                    if (!mbar_wait(smem_addr(&afull[slot]), (g / OZ_RING) & 1)) {
                        *vfail = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    oz_mma_slice<S, BN>(tmem, abase + slot * Cfg::A_BYTES, xbase + xb * Cfg::XBUF_BYTES, s, idesc,
                                        kt == 0);
                    umma_commit(smem_addr(&aempty[slot]));
                }
                umma_commit(smem_addr(&xempty[xb]));
            }
            umma_commit(smem_addr(&done));
        }
        __syncwarp();
    }
    if (!mbar_wait(smem_addr(&done), 0)) *vfail = 1;
    __syncthreads();
    if (*vfail) {
        if (threadIdx.x == 0) atomicOr(err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = m0 + warp * 32 + lane;
        const bool row_ok = r < Mvalid;
        const int em = row_ok ? row_exp[r >> 1] : 0;
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < BN; c += 16) {
            double acc[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = 0.0;
#pragma unroll
            for (int d = S - 1; d >= 0; --d) {  // smallest terms first
                uint32_t v[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(lane_base + (uint32_t)(d * BN + c)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const double w = ldexp(1.0, -7 * (d + 2));
#pragma unroll
                for (int i = 0; i < 16; ++i) acc[i] += w * (double)(int)v[i];
            }
            if (row_ok) {
                double bv[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int j = n0 + c + i;
                    bv[i] = j < Nvalid ? B[(int64_t)j * ldb_real + r] : 0.0;
                }
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int j = n0 + c + i;
                    if (j < Nvalid) {
                        const int fj = col_exp[j];
                        R[(int64_t)j * ldr_real + r] = (em == OZ_NONFINITE || fj == OZ_NONFINITE)
                                                           ? __longlong_as_double(0x7ff8000000000000LL)
                                                           : bv[i] - ldexp(acc[i], em + fj);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS)
                     : "memory");
    }
}
