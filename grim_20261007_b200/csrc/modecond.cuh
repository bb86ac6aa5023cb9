// 1-norm condition estimates of LU-factored systems, one CTA per system, no host
// synchronisation: the BoR per-mode condition gate (reference bor/factor.py:205-229,
// ModalFactor._condition: LAPACK zgecon on each mode's LU with the 1-norm of the mode
// matrix, the release limit applied by the caller).
//
// The estimate of ||inv(A)||_1 is Hager's method with Higham's refinements as LAPACK's
// zlacn2 runs it (N. J. Higham, ACM TOMS 14 (1988) 381-396, Algorithm 4.1): x = e/n, then
// at most four more rounds of an adjoint solve that picks the column e_j of largest |z_j|
// and a solve with e_j, stopping when the 1-norm stops growing or j repeats its modulus,
// and last the alternating-sign vector x_i = (-1)^i (1 + i/(n-1)) whose 2 ||inv(A) x||_1 / (3n)
// replaces the estimate when larger.  The operator is the one zgecon uses for a plain LU:
// inv(U) inv(L) without the row interchanges (inv(A) with its columns permuted, the same
// 1-norm), and inv(L^H) inv(U^H) for the adjoint.  A mirror-split mode is solved through
// its even and odd halves; its operator is the true inverse of the full matrix through
// them, inv(A) = S^T diag(inv(He), inv(Ho)) S with the orthogonal split S (the halves' row
// interchanges applied), adjoint S^T diag(inv(He)^H, inv(Ho)^H) S.
//
// Triangular solves: blocks of 32 rows, the coupling to solved blocks as a matrix-vector
// product over all 16 warps (coalesced column segments), the 32 x 32 diagonal block staged
// in shared memory and solved by one warp with shuffles.  Vectors live in global workspace
// (written by warp 0, read by all after a barrier: L1/L2 resident).
#pragma once
#include "common.cuh"

struct CondSysDev {
    int n, halves;
    int lu_c64[2];  // factor h stored in complex64
    int order[2];
    const void *lu[2];
    int64_t ld[2];
    const int *ipiv[2];
    int k, nfe, nfo;
    const int *p1, *p2, *fe, *fo;
    const double *s;
    const double2 *a;      // the full matrix (column-major), for ||A||_1
    int64_t lda;
    double *colsum;        // n column sums of |A|
    double2 *x, *w;        // n-element workspace vectors
};

constexpr int CS_THREADS = 512;
constexpr int CS_WARPS = CS_THREADS / 32;

struct CsShared {
    double2 red[CS_WARPS][33];  // per-warp partial products (+1 column against bank conflicts)
    double2 diag[32][33];       // diagonal block D[i][c]
    double rd[CS_WARPS];
    int ri[CS_WARPS];
    double scal[2];
    int sidx;
};

__device__ __forceinline__ double2 cs_ld(const double2 *p) { return *p; }
__device__ __forceinline__ double2 cs_ld(const float2 *p) { const float2 v = *p; return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 cs_conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cs_shfl(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ double2 cs_warp_sum(double2 v) {
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// D[i][c] = M[r0 + i, r0 + c] for i, c < nb (lane i, warps over c).
template <typename T>
__device__ __forceinline__ void cs_stage_diag(CsShared &sh, const T *M, int64_t ld, int r0, int nb) {
    const int i = threadIdx.x & 31;
    if (i < nb)
        for (int c = threadIdx.x >> 5; c < nb; c += CS_WARPS) sh.diag[i][c] = cs_ld(M + (int64_t)(r0 + c) * ld + r0 + i);
}

// x <- inv(L) x, L unit lower (strict lower part of the LU).
template <typename T>
__device__ void cs_lower(CsShared &sh, double2 *x, int n, const T *L, int64_t ld) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r0 = 0; r0 < n; r0 += 32) {
        const int nb = min(32, n - r0);
        double2 acc = make_double2(0.0, 0.0);
        if (lane < nb)
            for (int j = warp; j < r0; j += CS_WARPS) cfma(acc, cs_ld(L + (int64_t)j * ld + r0 + lane), x[j]);
        sh.red[warp][lane] = acc;
        cs_stage_diag(sh, L, ld, r0, nb);
        __syncthreads();
        if (warp == 0) {
            double2 v = make_double2(0.0, 0.0);
            if (lane < nb) {
                v = x[r0 + lane];
                for (int w = 0; w < CS_WARPS; ++w) v = csub(v, sh.red[w][lane]);
            }
            for (int c = 0; c < nb; ++c) {
                const double2 xc = cs_shfl(v, c);
                if (lane > c && lane < nb) cfms(v, sh.diag[lane][c], xc);
            }
            if (lane < nb) x[r0 + lane] = v;
        }
        __syncthreads();
    }
}

// x <- inv(U) x, U non-unit upper.
template <typename T>
__device__ void cs_upper(CsShared &sh, double2 *x, int n, const T *U, int64_t ld) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = (n + 31) / 32 - 1; b >= 0; --b) {
        const int r0 = b * 32, nb = min(32, n - r0), r1 = r0 + nb;
        double2 acc = make_double2(0.0, 0.0);
        if (lane < nb)
            for (int j = r1 + warp; j < n; j += CS_WARPS) cfma(acc, cs_ld(U + (int64_t)j * ld + r0 + lane), x[j]);
        sh.red[warp][lane] = acc;
        cs_stage_diag(sh, U, ld, r0, nb);
        __syncthreads();
        if (warp == 0) {
            double2 v = make_double2(0.0, 0.0);
            if (lane < nb) {
                v = x[r0 + lane];
                for (int w = 0; w < CS_WARPS; ++w) v = csub(v, sh.red[w][lane]);
            }
            for (int c = nb - 1; c >= 0; --c) {
                if (lane == c) v = cdiv(v, sh.diag[c][c]);
                const double2 xc = cs_shfl(v, c);
                if (lane < c) cfms(v, sh.diag[lane][c], xc);
            }
            if (lane < nb) x[r0 + lane] = v;
        }
        __syncthreads();
    }
}

// x <- inv(U^H) x (lower triangular, conjugated).
template <typename T>
__device__ void cs_upper_adj(CsShared &sh, double2 *x, int n, const T *U, int64_t ld) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r0 = 0; r0 < n; r0 += 32) {
        const int nb = min(32, n - r0);
        for (int c = warp; c < nb; c += CS_WARPS) {  // conj(U[0:r0, r0 + c]) . x[0:r0]
            double2 acc = make_double2(0.0, 0.0);
            const T *col = U + (int64_t)(r0 + c) * ld;
            for (int j = lane; j < r0; j += 32) cfma(acc, cs_conj(cs_ld(col + j)), x[j]);
            acc = cs_warp_sum(acc);
            if (lane == 0) sh.red[0][c] = acc;
        }
        cs_stage_diag(sh, U, ld, r0, nb);
        __syncthreads();
        if (warp == 0) {
            double2 v = make_double2(0.0, 0.0);
            if (lane < nb) v = csub(x[r0 + lane], sh.red[0][lane]);
            for (int c = 0; c < nb; ++c) {
                if (lane == c) v = cdiv(v, cs_conj(sh.diag[c][c]));
                const double2 xc = cs_shfl(v, c);
                if (lane > c && lane < nb) cfms(v, cs_conj(sh.diag[c][lane]), xc);
            }
            if (lane < nb) x[r0 + lane] = v;
        }
        __syncthreads();
    }
}

// x <- inv(L^H) x (upper triangular, unit, conjugated).
template <typename T>
__device__ void cs_lower_adj(CsShared &sh, double2 *x, int n, const T *L, int64_t ld) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = (n + 31) / 32 - 1; b >= 0; --b) {
        const int r0 = b * 32, nb = min(32, n - r0), r1 = r0 + nb;
        for (int c = warp; c < nb; c += CS_WARPS) {  // conj(L[r1:n, r0 + c]) . x[r1:n]
            double2 acc = make_double2(0.0, 0.0);
            const T *col = L + (int64_t)(r0 + c) * ld;
            for (int j = r1 + lane; j < n; j += 32) cfma(acc, cs_conj(cs_ld(col + j)), x[j]);
            acc = cs_warp_sum(acc);
            if (lane == 0) sh.red[0][c] = acc;
        }
        cs_stage_diag(sh, L, ld, r0, nb);
        __syncthreads();
        if (warp == 0) {
            double2 v = make_double2(0.0, 0.0);
            if (lane < nb) v = csub(x[r0 + lane], sh.red[0][lane]);
            for (int c = nb - 1; c >= 0; --c) {
                const double2 xc = cs_shfl(v, c);
                if (lane < c) cfms(v, cs_conj(sh.diag[c][lane]), xc);
            }
            if (lane < nb) x[r0 + lane] = v;
        }
        __syncthreads();
    }
}

// Row interchanges of an LU (1-based ipiv): forward (before the L solve) or backward
// (after the adjoint's L^H solve).  One thread; the caller's barrier follows.
__device__ void cs_swaps(double2 *x, int n, const int *ipiv, bool forward) {
    if (threadIdx.x != 0) return;
    for (int t = 0; t < n; ++t) {
        const int i = forward ? t : n - 1 - t;
        const int p = ipiv[i] - 1;
        if (p != i && p >= 0 && p < n) {
            const double2 a = x[i];
            x[i] = x[p];
            x[p] = a;
        }
    }
}

template <typename T>
__device__ void cs_apply_lu_t(CsShared &sh, double2 *x, int n, const T *lu, int64_t ld, const int *ipiv, bool adjoint) {
    if (!adjoint) {
        if (ipiv) {
            cs_swaps(x, n, ipiv, true);
            __syncthreads();
        }
        cs_lower(sh, x, n, lu, ld);
        cs_upper(sh, x, n, lu, ld);
    } else {
        cs_upper_adj(sh, x, n, lu, ld);
        cs_lower_adj(sh, x, n, lu, ld);
        if (ipiv) {
            cs_swaps(x, n, ipiv, false);
            __syncthreads();
        }
    }
}

__device__ void cs_apply_lu(CsShared &sh, double2 *x, int n, const void *lu, bool c64, int64_t ld, const int *ipiv,
                            bool adjoint) {
    if (c64) cs_apply_lu_t(sh, x, n, (const float2 *)lu, ld, ipiv, adjoint);
    else cs_apply_lu_t(sh, x, n, (const double2 *)lu, ld, ipiv, adjoint);
}

// x <- inv(A) x or inv(A)^H x for one system (see the header).
__device__ void cs_apply(CsShared &sh, const CondSysDev &S, bool adjoint) {
    if (!S.halves) {
        cs_apply_lu(sh, S.x, S.n, S.lu[0], S.lu_c64[0], S.ld[0], nullptr, adjoint);
        return;
    }
    const double r = 0.7071067811865475244;
    const int k = S.k, ke = S.order[0], ko = S.order[1];
    double2 *xe = S.w, *xo = S.w + ke;
    for (int i = threadIdx.x; i < max(ke, ko); i += blockDim.x) {
        if (i < k) {
            const double2 a = S.x[S.p1[i]], b = S.x[S.p2[i]];
            const double s = S.s[i];
            xe[i] = make_double2(r * (a.x + s * b.x), r * (a.y + s * b.y));
            xo[i] = make_double2(r * (a.x - s * b.x), r * (a.y - s * b.y));
        } else {
            if (i < ke) xe[i] = S.x[S.fe[i - k]];
            if (i < ko) xo[i] = S.x[S.fo[i - k]];
        }
    }
    __syncthreads();
    cs_apply_lu(sh, xe, ke, S.lu[0], S.lu_c64[0], S.ld[0], S.ipiv[0], adjoint);
    cs_apply_lu(sh, xo, ko, S.lu[1], S.lu_c64[1], S.ld[1], S.ipiv[1], adjoint);
    for (int i = threadIdx.x; i < max(ke, ko); i += blockDim.x) {
        if (i < k) {
            const double2 e = xe[i], o = xo[i];
            const double rs = r * S.s[i];
            S.x[S.p1[i]] = make_double2(r * (e.x + o.x), r * (e.y + o.y));
            S.x[S.p2[i]] = make_double2(rs * (e.x - o.x), rs * (e.y - o.y));
        } else {
            if (i < ke) S.x[S.fe[i - k]] = xe[i];
            if (i < ko) S.x[S.fo[i - k]] = xo[i];
        }
    }
    __syncthreads();
}

// sum_i |x_i| (in a fixed order), and x_i <- x_i / |x_i| (1 where |x_i| <= the safe
// minimum) when sign; the result is read by every thread.
__device__ double cs_norm1(CsShared &sh, double2 *x, int n, bool sign) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double2 v = x[i];
        const double a = hypot(v.x, v.y);
        s += a;
        if (sign) x[i] = a > 2.2250738585072014e-308 ? make_double2(v.x / a, v.y / a) : make_double2(1.0, 0.0);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh.rd[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < CS_WARPS; ++w) t += sh.rd[w];
        sh.scal[0] = t;
    }
    __syncthreads();
    const double out = sh.scal[0];
    __syncthreads();
    return out;
}

// First index of the largest |x_i|; every thread gets it.
__device__ int cs_argmax(CsShared &sh, const double2 *x, int n) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double best = -1.0;
    int bi = n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = hypot(x[i].x, x[i].y);
        if (a > best) { best = a; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (lane == 0) { sh.rd[warp] = best; sh.ri[warp] = bi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = -1.0;
        int j = n;
        for (int w = 0; w < CS_WARPS; ++w)
            if (sh.rd[w] > b || (sh.rd[w] == b && sh.ri[w] < j)) { b = sh.rd[w]; j = sh.ri[w]; }
        sh.sidx = j < n ? j : 0;
    }
    __syncthreads();
    const int out = sh.sidx;
    __syncthreads();
    return out;
}

// column sums of |A| for every system: grid (ceil(nmax / 8), count), 256 threads, a warp
// per column.
__global__ void __launch_bounds__(256) k_cond_colsum(const CondSysDev *systems) {
    const CondSysDev &S = systems[blockIdx.y];
    const int lane = threadIdx.x & 31, j = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (j >= S.n) return;
    const double2 *a = S.a + (int64_t)j * S.lda;
    double s = 0.0;
    for (int i = lane; i < S.n; i += 32) s += hypot(a[i].x, a[i].y);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) S.colsum[j] = s;
}

__device__ double cs_estimate(CsShared &sh, const CondSysDev &S) {
    const int n = S.n;
    double2 *x = S.x;
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = make_double2(1.0 / n, 0.0);
    __syncthreads();
    cs_apply(sh, S, false);
    if (n == 1) return hypot(x[0].x, x[0].y);
    double est = cs_norm1(sh, x, n, true);
    cs_apply(sh, S, true);
    int j = cs_argmax(sh, x, n);
    for (int iter = 2;; ++iter) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = make_double2(i == j ? 1.0 : 0.0, 0.0);
        __syncthreads();
        cs_apply(sh, S, false);
        const double old = est;
        est = cs_norm1(sh, x, n, true);
        if (est <= old) break;  // the 1-norm stopped growing
        cs_apply(sh, S, true);
        const int jlast = j;
        j = cs_argmax(sh, x, n);
        const double zl = hypot(x[jlast].x, x[jlast].y), zj = hypot(x[j].x, x[j].y);
        __syncthreads();
        if (!(zl != zj && iter < 5)) break;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        x[i] = make_double2((i & 1 ? -1.0 : 1.0) * (1.0 + (double)i / (double)(n - 1)), 0.0);
    __syncthreads();
    cs_apply(sh, S, false);
    const double alt = 2.0 * (cs_norm1(sh, x, n, false) / (3.0 * n));
    return alt > est ? alt : est;
}

// cond[s] = ||A_s||_1 * est ||inv(A_s)||_1 (NaN when the system holds a NaN; inf when the
// estimate or the norm is zero or overflows, zgecon's rcond = 0).  One CTA per system.
__global__ void __launch_bounds__(CS_THREADS) k_cond_lacn2(const CondSysDev *systems, double *cond) {
    __shared__ CsShared sh;
    __shared__ CondSysDev S;
    if (threadIdx.x == 0) S = systems[blockIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double an = 0.0;
    for (int j = threadIdx.x; j < S.n; j += blockDim.x) {
        const double c = S.colsum[j];
        an = (c > an || c != c) ? c : an;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_down_sync(0xffffffffu, an, o);
        an = (v > an || v != v) ? v : an;
    }
    if (lane == 0) sh.rd[warp] = an;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < CS_WARPS; ++w) m = (sh.rd[w] > m || sh.rd[w] != sh.rd[w]) ? sh.rd[w] : m;
        sh.scal[1] = m;
    }
    __syncthreads();
    an = sh.scal[1];
    __syncthreads();
    const double est = cs_estimate(sh, S);
    if (threadIdx.x == 0) {
        double c;
        if (an != an || est != est) c = NAN;
        else if (!(an > 0.0) || !(est > 0.0)) c = INFINITY;
        else c = 1.0 / ((1.0 / est) / an);
        cond[blockIdx.x] = c;
    }
}
