// Dense complex LU (getrf) and multi-RHS triangular solves (getrs) on column-major
// complex128 / complex64 matrices, SIMT kernels.
//
// Factorization (right-looking, block width NB = 64), three launches per panel j:
//   k_diag_lu     one CTA: unpivoted LU of the NB x NB diagonal block in shared memory,
//                 the diagonal-pivot certificate inside it, and inv(L11), inv(U11) by a
//                 blocked recursive inversion (8 x 8 leaves per warp, then 16, 32, 64);
//   k_panel_apply one CTA per 64-row strip of A21 (L21 = A21 inv(U11), certificate
//                 |l_ic u_cc|_1 <= |u_cc|_1) and per 64-column strip of A12
//                 (U12 = inv(L11) A12), both with backups; the last CTA to finish
//                 refactors the panel with partial pivoting if any certificate failed;
//   k_gemm_rt     A22 -= L21 U12.
// Static pivoting (no_fallback): the certificate is still computed but never acted on, so
// the factors are the unpivoted ones; callers that ask for it check the solution's
// backward error and refactor with partial pivoting when it fails (grim_zgesv_guarded).
// Partial pivoting picks the diagonal at step c exactly when |a_ic^(c)|_1 <= |a_cc^(c)|_1
// for every i > c (LAPACK izamax: |re|+|im|, first index on ties), and a_ic^(c) = l_ic u_cc,
// so a passing certificate proves the unpivoted factors equal getrf's
// (reference linalg/dense.py:114-155 via scipy.linalg.lu_factor).
#pragma once
#include "common.cuh"
#include "tc_gemm.cuh"

// Tensor-core operands of the trailing update written by the complex64 panel solve itself
// (tile layout of tc_gemm.cuh): L21 as the A operand (real rows 2m, 2m+1 of trailing row
// m, a_rows rows) and U12 as the B operand (row = trailing column, b_rows rows), both with
// 2 NB real columns, split into TF32 hi and lo.  a_hi == nullptr: not wanted.
struct PanelPack {
    float *a_hi = nullptr, *a_lo = nullptr;
    int a_rows = 0;
    float *b_hi = nullptr, *b_lo = nullptr;
    int b_rows = 0;
};

__device__ __forceinline__ void pack_pair(float *hi, float *lo, int64_t off, float x0, float x1) {
    const float h0 = tf32_rna(x0), h1 = tf32_rna(x1);
    *reinterpret_cast<float2 *>(hi + off) = make_float2(h0, h1);
    *reinterpret_cast<float2 *>(lo + off) = make_float2(tf32_rna(x0 - h0), tf32_rna(x1 - h1));
}

#define NB 64
#define RT_BM 64
#define RT_BN 128
#define RT_BK 8
#define RT_THREADS 256

// ------------------------------------------------------------------ register-tiled GEMM
// C[MxN] = (BETA ? C : 0) + (NEG ? -1 : 1) * A[MxK] * B[KxN], column-major, ACC arithmetic.
// 64 x 128 CTA tile, 256 threads each owning 4 x 8 outputs, two shared-memory stages
// filled through registers.
// Batched over blockIdx.z: operand z starts sA / sB / sC elements after operand 0.
template <typename ACC, typename TA, typename TB, typename TC, bool NEG, bool BETA>
__global__ void __launch_bounds__(RT_THREADS)
k_gemm_rt(int M, int N, int K, const TA *__restrict__ A, int64_t lda, const TB *__restrict__ B, int64_t ldb,
          TC *__restrict__ C, int64_t ldc, int64_t sA, int64_t sB, int64_t sC) {
    using R = typename real_of<ACC>::type;
    A += blockIdx.z * sA;
    B += blockIdx.z * sB;
    C += blockIdx.z * sC;
    __shared__ ACC As[2][RT_BK][RT_BM];
    __shared__ ACC Bs[2][RT_BK][RT_BN];
    const int t = threadIdx.x;
    const int tx = t & 15, ty = t >> 4;
    const int m0 = blockIdx.x * RT_BM, n0 = blockIdx.y * RT_BN;
    ACC acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = czero<ACC>();
    ACC ra[2], rb[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int e = t + RT_THREADS * i;
            const int r = e & 63, c = e >> 6;
            const int gm = m0 + r, gk = k0 + c;
            ACC v = czero<ACC>();
            if (gm < M && gk < K) {
                const TA x = A[(int64_t)gk * lda + gm];
                v = mk((R)x.x, (R)x.y);
            }
            ra[i] = v;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = t + RT_THREADS * i;
            const int r = e & 7, c = e >> 3;
            const int gk = k0 + r, gn = n0 + c;
            ACC v = czero<ACC>();
            if (gk < K && gn < N) {
                const TB x = B[(int64_t)gn * ldb + gk];
                v = mk((R)x.x, (R)x.y);
            }
            rb[i] = v;
        }
    };
    auto store = [&](int s) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int e = t + RT_THREADS * i;
            As[s][e >> 6][e & 63] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = t + RT_THREADS * i;
            Bs[s][e & 7][e >> 3] = rb[i];
        }
    };
    const int nk = (K + RT_BK - 1) / RT_BK;
    load(0);
    store(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int cur = kt & 1;
        if (kt + 1 < nk) load((kt + 1) * RT_BK);
#pragma unroll
        for (int kk = 0; kk < RT_BK; ++kk) {
            ACC a[4], b[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[cur][kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[cur][kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) cfma(acc[i][j], a[i], b[j]);
        }
        if (kt + 1 < nk) store(cur ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + tx + 16 * i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int gn = n0 + ty + 16 * j;
            if (gn >= N) continue;
            TC *p = C + (int64_t)gn * ldc + gm;
            ACC v = acc[i][j];
            if (NEG) v = mk(-v.x, -v.y);
            if (BETA) {
                const TC o = *p;
                v.x += (R)o.x;
                v.y += (R)o.y;
            }
            TC w;
            w.x = (decltype(w.x))v.x;
            w.y = (decltype(w.y))v.y;
            *p = w;
        }
    }
}

// ------------------------------------------------------------------ small-block helpers
template <typename C>
__device__ __forceinline__ C one_c() {
    return mk((typename real_of<C>::type)1, (typename real_of<C>::type)0);
}

// Padded leading dimension of 64 x 64 triangular blocks in shared memory: row r, column c
// at [c * NBP + r]; the odd padding keeps the four sub-lanes of a substitution on
// distinct banks.
#define NBP 65

template <typename C>
__device__ __forceinline__ C shfl_xor_c(C v, int m) {
    v.x = __shfl_xor_sync(0xffffffffu, v.x, m);
    v.y = __shfl_xor_sync(0xffffffffu, v.y, m);
    return v;
}
template <typename C>
__device__ __forceinline__ C shfl_c(C v, int src) {
    v.x = __shfl_sync(0xffffffffu, v.x, src);
    v.y = __shfl_sync(0xffffffffu, v.y, src);
    return v;
}
template <typename C>
__device__ __forceinline__ C reduce4(C v) {
    C o = shfl_xor_c(v, 1);
    v.x += o.x;
    v.y += o.y;
    o = shfl_xor_c(v, 2);
    v.x += o.x;
    v.y += o.y;
    return v;
}

// Substitutions on one 64-long vector, shared by 4 consecutive lanes (sub-lane s owns
// the entries p = 4 i + s, i < 16, in registers v[i]).  T is a 64 x 64 block in smem
// (leading dim NBP), rd[c] = 1 / T(c, c).  Fully unrolled so v[] stays in registers.
//
// row_upper:   x T = a  (x a row vector, T upper)      x_c = (a_c - sum_{p<c} x_p T_pc) rd_c
// col_lower1:  T x = a  (T unit lower)                 x_r = a_r - sum_{p<r} T_rp x_p
// col_upper:   T x = a  (T upper)                      x_r = (a_r - sum_{p>r} T_rp x_p) rd_r
template <typename C>
__device__ __forceinline__ void subst_row_upper(C (&v)[16], const C *T, const C *rd, int nbj, int s) {
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        if (c < nbj) {
            C part = czero<C>();
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (4 * i + s < c) cfma(part, v[i], T[c * NBP + 4 * i + s]);
            part = reduce4(part);
            if (s == (c & 3)) v[c >> 2] = cmul(csub(v[c >> 2], part), rd[c]);
        }
    }
}
template <typename C>
__device__ __forceinline__ void subst_col_lower1(C (&v)[16], const C *T, int nbj, int s) {
#pragma unroll
    for (int r = 0; r < NB; ++r) {
        if (r < nbj) {
            C part = czero<C>();
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (4 * i + s < r) cfma(part, T[(4 * i + s) * NBP + r], v[i]);
            part = reduce4(part);
            if (s == (r & 3)) v[r >> 2] = csub(v[r >> 2], part);
        }
    }
}
template <typename C>
__device__ __forceinline__ void subst_col_upper(C (&v)[16], const C *T, const C *rd, int nbj, int s) {
#pragma unroll
    for (int r = NB - 1; r >= 0; --r) {
        if (r < nbj) {
            C part = czero<C>();
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (4 * i + s > r && 4 * i + s < nbj) cfma(part, T[(4 * i + s) * NBP + r], v[i]);
            part = reduce4(part);
            if (s == (r & 3)) v[r >> 2] = cmul(csub(v[r >> 2], part), rd[r]);
        }
    }
}

// x U = a for one 64-long row vector shared by 4 consecutive lanes (sub-lane s owns the
// entries p = 4 i + s, i < 16, in v[i]; T is U in shared memory, leading dim NBP, rd its
// reciprocal diagonal, entries past nbj zero with rd = 1).  The same result as
// subst_row_upper, computed right-looking as a loop whose body stays in the instruction
// cache: each column's value, once final, is broadcast to the group and subtracted from the
// later entries; after each block of four columns the pending entries shift down one
// register and the solved ones into x, so every register index is a compile-time constant.
// Phase p (blocks 4 p .. 4 p + 3) keeps 16 - 4 p pending registers.
template <typename C, int LIVE>
__device__ __forceinline__ void subst_row_upper_blocks(C (&v)[16], C (&x)[16], const C *T, const C *rd, int nbj,
                                                       int s, int b0) {
    const int base = (int)(threadIdx.x & 31u) & ~3;
#pragma unroll 1
    for (int b = b0; b < b0 + 4; ++b) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
            const int c = 4 * b + cc;
            C xc = czero<C>();
            if (s == cc && c < nbj) xc = cmul(v[0], rd[c]);
            xc = shfl_c(xc, base | cc);
            if (s == cc) v[0] = xc;
            if (s > cc) cfms(v[0], xc, T[(4 * b + s) * NBP + c]);
#pragma unroll
            for (int i = 1; i < LIVE; ++i)
                if (b + i < 16) cfms(v[i], xc, T[(4 * (b + i) + s) * NBP + c]);
        }
#pragma unroll
        for (int i = 0; i + 1 < 16; ++i) x[i] = x[i + 1];
        x[15] = v[0];
#pragma unroll
        for (int i = 0; i + 1 < LIVE; ++i) v[i] = v[i + 1];
        v[LIVE - 1] = czero<C>();
    }
}

template <typename C>
__device__ __forceinline__ void subst_row_upper_loop(C (&v)[16], const C *T, const C *rd, int nbj, int s) {
    C x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = czero<C>();
    subst_row_upper_blocks<C, 16>(v, x, T, rd, nbj, s, 0);
    subst_row_upper_blocks<C, 12>(v, x, T, rd, nbj, s, 4);
    subst_row_upper_blocks<C, 8>(v, x, T, rd, nbj, s, 8);
    subst_row_upper_blocks<C, 4>(v, x, T, rd, nbj, s, 12);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = x[i];
}

// T x = a (T unit lower) for one 64-long column vector shared by 4 lanes, the same result
// as subst_col_lower1, right-looking in a loop whose body stays in the instruction cache:
// entry r, once final, is broadcast to the group and subtracted from the later entries;
// after each block of four entries the pending ones shift down a register and the solved
// ones into x.  Phase p (blocks 4 p .. 4 p + 3) keeps 16 - 4 p pending registers.
template <typename C, int LIVE>
__device__ __forceinline__ void subst_col_lower1_blocks(C (&v)[16], C (&x)[16], const C *T, int s, int b0) {
    const int base = (int)(threadIdx.x & 31u) & ~3;
#pragma unroll 1
    for (int b = b0; b < b0 + 4; ++b) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
            const int r = 4 * b + cc;
            const C xr = shfl_c(v[0], base | cc);
            if (s > cc) cfms(v[0], xr, T[r * NBP + 4 * b + s]);
#pragma unroll
            for (int i = 1; i < LIVE; ++i)
                if (b + i < 16) cfms(v[i], xr, T[r * NBP + 4 * (b + i) + s]);
        }
#pragma unroll
        for (int i = 0; i + 1 < 16; ++i) x[i] = x[i + 1];
        x[15] = v[0];
#pragma unroll
        for (int i = 0; i + 1 < LIVE; ++i) v[i] = v[i + 1];
        v[LIVE - 1] = czero<C>();
    }
}
template <typename C>
__device__ __forceinline__ void subst_col_lower1_loop(C (&v)[16], const C *T, int s) {
    C x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = czero<C>();
    subst_col_lower1_blocks<C, 16>(v, x, T, s, 0);
    subst_col_lower1_blocks<C, 12>(v, x, T, s, 4);
    subst_col_lower1_blocks<C, 8>(v, x, T, s, 8);
    subst_col_lower1_blocks<C, 4>(v, x, T, s, 12);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = x[i];
}

// T x = a (T upper, rd its reciprocal diagonal), the same result as subst_col_upper,
// right-looking from the last entry down: the block being solved sits in v[15], pending
// entries below it, and after each block everything shifts up a register (the solved entry
// into x from the bottom).  Phase p (blocks 15 - 4 p .. 12 - 4 p) keeps 16 - 4 p registers.
template <typename C, int LIVE>
__device__ __forceinline__ void subst_col_upper_blocks(C (&v)[16], C (&x)[16], const C *T, const C *rd, int s,
                                                       int b0) {
    const int base = (int)(threadIdx.x & 31u) & ~3;
#pragma unroll 1
    for (int b = b0; b > b0 - 4; --b) {
#pragma unroll
        for (int cc = 3; cc >= 0; --cc) {
            const int r = 4 * b + cc;
            C xr = czero<C>();
            if (s == cc) xr = cmul(v[15], rd[r]);
            xr = shfl_c(xr, base | cc);
            if (s == cc) v[15] = xr;
            if (s < cc) cfms(v[15], xr, T[r * NBP + 4 * b + s]);
#pragma unroll
            for (int i = 16 - LIVE; i < 15; ++i)
                if (b - 15 + i >= 0) cfms(v[i], xr, T[r * NBP + 4 * (b - 15 + i) + s]);
        }
#pragma unroll
        for (int i = 15; i > 0; --i) x[i] = x[i - 1];
        x[0] = v[15];
#pragma unroll
        for (int i = 15; i > 16 - LIVE; --i) v[i] = v[i - 1];
        v[16 - LIVE] = czero<C>();
    }
}
template <typename C>
__device__ __forceinline__ void subst_col_upper_loop(C (&v)[16], const C *T, const C *rd, int s) {
    C x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = czero<C>();
    subst_col_upper_blocks<C, 16>(v, x, T, rd, s, 15);
    subst_col_upper_blocks<C, 12>(v, x, T, rd, s, 11);
    subst_col_upper_blocks<C, 8>(v, x, T, rd, s, 7);
    subst_col_upper_blocks<C, 4>(v, x, T, rd, s, 3);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = x[i];
}

// Stage the nbj x nbj diagonal block at (j, j) into smem T (padded, zero outside) and
// the reciprocals of its diagonal into rd (1 outside).
// Sixteen loads per thread are in flight before their stores: a 64-thread CTA stages the
// block in four round trips to memory instead of sixty-four.
template <typename C>
__device__ __forceinline__ void stage_diag(const C *A, int64_t lda, int j, int nbj, C *T, C *rd) {
    constexpr int U = 16;
    for (int e0 = threadIdx.x; e0 < NB * NB; e0 += U * blockDim.x) {
        C x[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * (int)blockDim.x;
            const int r = e & 63, c = e >> 6;
            x[u] = (e < NB * NB && r < nbj && c < nbj) ? A[(int64_t)(j + c) * lda + j + r] : czero<C>();
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * (int)blockDim.x;
            if (e < NB * NB) T[(e >> 6) * NBP + (e & 63)] = x[u];
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < NB; r += blockDim.x) rd[r] = r < nbj ? crecip(T[r * NBP + r]) : one_c<C>();
    __syncthreads();
}

// ------------------------------------------------------------------ diagonal block
// Runtime-indexed read / write of a small register array through a static select chain
// (keeps the array in registers).
template <typename C, int L>
__device__ __forceinline__ C vget(const C (&v)[L], int idx) {
    C x = czero<C>();
#pragma unroll
    for (int i = 0; i < L; ++i)
        if (i == idx) x = v[i];
    return x;
}
template <typename C, int L>
__device__ __forceinline__ void vset(C (&v)[L], int idx, C x) {
#pragma unroll
    for (int i = 0; i < L; ++i)
        if (i == idx) v[i] = x;
}

// One CTA of 256 threads: unpivoted right-looking LU of the nbj x nbj diagonal block
// (nbj <= 64), the diagonal-pivot certificate, a backup of the block and identity ipiv
// entries.  Warp w owns rows 32 (w / 4) + lane and columns 16 (w % 4) .. + 15 in
// registers, so that a warp whose rows or columns are all factored skips a step as a
// whole.  The column loop is split into 4 groups of 16 with the inner 16 unrolled, so
// every register index is a compile-time constant.  Step k (two barriers; shared buffers
// double-buffered by step parity):
//   the owners of row k publish it;
//   the warps holding column k form l_rk = a_rk / a_kk for their rows r > k;
//   every warp with rows and columns beyond k applies a_rc -= l_rk a_kc.
// Certificate: |a_rk^(k)|_1 <= |a_kk^(k)|_1 for r > k, and a_kk != 0.
template <typename C>
__device__ __forceinline__ void diag_lu_cta(int n, C *A, int64_t lda, int j, int nbj, C *backup_col, int *cert,
                                            int *ipiv) {
    __shared__ C rowbuf[2][NB];
    __shared__ C lbuf[2][NB];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int h = warp >> 2, g = warp & 3, r = 32 * h + lane, c0 = 16 * g;
    C v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int c = c0 + i;
        C x = czero<C>();
        if (r < nbj && c < nbj) {
            x = A[(int64_t)(j + c) * lda + j + r];
            backup_col[(int64_t)c * n + r] = x;
        }
        v[i] = x;
    }
    if (t < nbj) ipiv[j + t] = j + t + 1;
    int bad = 0;
    const int nkg = (nbj + 15) >> 4;
#pragma unroll 1
    for (int kg = 0; kg < nkg; ++kg) {
#pragma unroll
        for (int ik = 0; ik < 16; ++ik) {
            const int k = 16 * kg + ik;
            if (k >= nbj) break;
            const int buf = k & 1;
            if (r == k) {
#pragma unroll
                for (int i = 0; i < 16; ++i) rowbuf[buf][c0 + i] = v[i];
            }
            __syncthreads();
            const bool rows_left = 32 * h + 31 > k;
            const bool below = r > k && r < nbj;
            if (g == kg && rows_left) {
                const C piv = rowbuf[buf][k];
                if (r == k && cabs1(piv) == 0) bad = 1;
                if (below) {
                    const C a = v[ik];
                    if (!(cabs1(a) <= cabs1(piv))) bad = 1;
                    v[ik] = cmul(a, crecip(piv));
                    lbuf[buf][r] = v[ik];
                }
            }
            __syncthreads();
            if (rows_left && below) {
                if (g > kg) {
                    const C l = lbuf[buf][r];
                    const C *u = rowbuf[buf] + c0;
#pragma unroll
                    for (int i = 0; i < 16; ++i) cfms(v[i], l, u[i]);
                } else if (g == kg) {
                    const C l = v[ik];
                    const C *u = rowbuf[buf] + c0;
#pragma unroll
                    for (int i = ik + 1; i < 16; ++i) cfms(v[i], l, u[i]);
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int c = c0 + i;
        if (r < nbj && c < nbj) A[(int64_t)(j + c) * lda + j + r] = v[i];
    }
    if (__syncthreads_or(bad) && t == 0) atomicOr(cert, 1);
}

template <typename C>
__global__ void __launch_bounds__(256)
k_diag_lu(int n, C *A, int64_t lda, int j, int nbj, C *backup_col, int *cert, int *ipiv) {
    diag_lu_cta<C>(n, A, lda, j, nbj, backup_col, cert, ipiv);
}

// ------------------------------------------------------------------ pivoted panel (fallback)
// Executed by one CTA (256 threads) after restoring the panel: LAPACK getf2 on the
// (n - j) x nbj panel in global memory, then row interchanges and U12 = inv(L11) A12
// (forward substitution) on every trailing column.
template <typename C>
__device__ void pivoted_panel(int n, C *A, int64_t lda, int j, int nbj, int *ipiv, int *info, int *swapped) {
    using R = typename real_of<C>::type;
    __shared__ R wv[8];
    __shared__ int wi[8];
    __shared__ int s_piv, s_any;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_any = 0;
    __syncthreads();
    for (int kk = 0; kk < nbj; ++kk) {
        const int col = j + kk;
        R best = (R)-1;
        int bi = 0x7fffffff;
        for (int r = col + t; r < n; r += 256) {
            const R v = cabs1(A[(int64_t)col * lda + r]);
            if (v > best || (v == best && r < bi)) { best = v; bi = r; }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const R ov = __shfl_down_sync(0xffffffffu, best, off);
            const int oi = __shfl_down_sync(0xffffffffu, bi, off);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { wv[warp] = best; wi[warp] = bi; }
        __syncthreads();
        if (t == 0) {
            best = wv[0];
            bi = wi[0];
            for (int w = 1; w < 8; ++w)
                if (wv[w] > best || (wv[w] == best && wi[w] < bi)) { best = wv[w]; bi = wi[w]; }
            s_piv = bi;
            ipiv[col] = bi + 1;
            if (bi != col) s_any = 1;
        }
        __syncthreads();
        const int p = s_piv;
        const C pv = A[(int64_t)col * lda + p];
        const bool zero = (pv.x == 0 && pv.y == 0);
        if (zero) {
            if (t == 0 && *info == 0) *info = col + 1;
        } else if (p != col) {
            for (int c = t; c < n; c += 256) {  // whole rows from column j on
                if (c < j) continue;
                C *a = A + (int64_t)c * lda;
                const C x = a[col];
                a[col] = a[p];
                a[p] = x;
            }
        }
        __syncthreads();
        if (!zero) {
            const C d = A[(int64_t)col * lda + col];
            for (int r = col + 1 + t; r < n; r += 256) A[(int64_t)col * lda + r] = cdiv(A[(int64_t)col * lda + r], d);
        }
        __syncthreads();
        for (int r = col + 1 + t; r < n; r += 256) {
            const C l = A[(int64_t)col * lda + r];
            for (int c = kk + 1; c < nbj; ++c) cfms(A[(int64_t)(j + c) * lda + r], l, A[(int64_t)(j + c) * lda + col]);
        }
        __syncthreads();
    }
    // U12 = inv(L11) A12 by forward substitution, one thread per trailing column
    for (int c = j + nbj + t; c < n; c += 256) {
        C *a = A + (int64_t)c * lda;
        for (int i = 1; i < nbj; ++i) {
            C acc = a[j + i];
            for (int p = 0; p < i; ++p) cfms(acc, A[(int64_t)(j + p) * lda + j + i], a[j + p]);
            a[j + i] = acc;
        }
    }
    if (t == 0) *swapped = s_any;
}


// ------------------------------------------------------------------ panel apply
// nblocks = nL + nU CTAs of 256 threads; this is CTA b.  CTA b < nL: 64 rows of A21 (4
// lanes per row), L21 = A21 inv(U11) by row substitution, certificate
// |l_ic u_cc|_1 <= |u_cc|_1.  CTA b >= nL: 64 columns of A12, U12 = inv(L11) A12 by column
// substitution.  Both back up what they overwrite; the last CTA to finish runs the
// pivoted refactorization when any certificate failed.  Dynamic smem: NB * NBP + NB
// elements.
template <typename C>
__device__ __forceinline__ void panel_apply_cta(int n, C *A, int64_t lda, int j, int nbj, int nL, int b, int nblocks,
                                                C *backup_col, C *backup_row, int *cert, int *counter, int *swapped,
                                                int *ipiv, int *info, int *pivoted, PanelPack pk = PanelPack(),
                                                int no_fallback = 0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *T = reinterpret_cast<C *>(smem_raw);
    C *rd = T + NB * NBP;
    const int t = threadIdx.x, s = t & 3, lane_vec = t >> 2;
    const bool is_l = b < nL;
    stage_diag(A, lda, j, nbj, T, rd);
    C v[16];
    int bad = 0;
    if (is_l) {
        const int row = j + nbj + NB * b + lane_vec;
        const bool ok = row < n;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int c = 4 * i + s;
            C x = czero<C>();
            if (ok && c < nbj) {
                x = A[(int64_t)(j + c) * lda + row];
                backup_col[(int64_t)c * n + (row - j)] = x;
            }
            v[i] = x;
        }
        subst_row_upper_loop(v, T, rd, nbj, s);
        if (ok) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int c = 4 * i + s;
                if (c < nbj) {
                    const C ucc = T[c * NBP + c];
                    if (!(cabs1(cmul(v[i], ucc)) <= cabs1(ucc))) bad = 1;
                    A[(int64_t)(j + c) * lda + row] = v[i];
                }
            }
        }
        if constexpr (sizeof(C) == sizeof(float2)) {
            if (pk.a_hi) {  // rows past the matrix are written as zero padding
                const int m = NB * b + lane_vec;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int c = 4 * i + s;
                    const float xr = ok ? (float)v[i].x : 0.f, xi = ok ? (float)v[i].y : 0.f;
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * m, 2 * c, pk.a_rows), xr, -xi);
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * m + 1, 2 * c, pk.a_rows), xi, xr);
                }
            }
        }
    } else {
        const int col = j + nbj + NB * (b - nL) + lane_vec;
        const bool ok = col < n;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = 4 * i + s;
            C x = czero<C>();
            if (ok && r < nbj) {
                x = A[(int64_t)col * lda + j + r];
                backup_row[(int64_t)(col - j - nbj) * NB + r] = x;
            }
            v[i] = x;
        }
        subst_col_lower1_loop(v, T, s);
        if (ok) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int r = 4 * i + s;
                if (r < nbj) A[(int64_t)col * lda + j + r] = v[i];
            }
        }
        if constexpr (sizeof(C) == sizeof(float2)) {
            if (pk.a_hi) {
                const int nb_row = NB * (b - nL) + lane_vec;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int r = 4 * i + s;
                    pack_pair(pk.b_hi, pk.b_lo, tc_tile_offset(nb_row, 2 * r, pk.b_rows), ok ? (float)v[i].x : 0.f,
                              ok ? (float)v[i].y : 0.f);
                }
            }
        }
    }
    if (__syncthreads_or(bad) && t == 0) atomicOr(cert, 1);
    // last CTA: pivoted fallback if any certificate failed
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (t == 0) s_last = (atomicAdd(counter, 1) == nblocks - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (no_fallback || atomicAdd(cert, 0) == 0) return;
    for (int c = 0; c < nbj; ++c)
        for (int r = t; r < n - j; r += 256) A[(int64_t)(j + c) * lda + j + r] = backup_col[(int64_t)c * n + r];
    for (int c = j + nbj; c < n; ++c)
        for (int r = t; r < nbj; r += 256) A[(int64_t)c * lda + j + r] = backup_row[(int64_t)(c - j - nbj) * NB + r];
    __syncthreads();
    pivoted_panel(n, A, lda, j, nbj, ipiv, info, swapped);
    if (t == 0) atomicAdd(pivoted, 1);
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (pk.a_hi) {  // the refactored panel: pack both operands again (this CTA alone)
            __syncthreads();
            const int rest = n - j - nbj;
            const float2 *Af = reinterpret_cast<const float2 *>(A);
            for (int64_t e = t; e < (int64_t)pk.a_rows * (2 * NB / 4); e += 256)
                tc_pack_a_chunk(e, rest, nbj, Af + (int64_t)j * lda + j + nbj, lda, pk.a_hi, pk.a_lo, pk.a_rows,
                                pk.a_rows, 0, 2 * NB, 1.f);
            for (int64_t e = t; e < (int64_t)pk.b_rows * (2 * NB / 4); e += 256)
                tc_pack_b_chunk(e, nbj, rest, Af + (int64_t)(j + nbj) * lda + j, lda, pk.b_hi, pk.b_lo, pk.b_rows,
                                2 * NB);
        }
    }
}

template <typename C>
__global__ void __launch_bounds__(256)
k_panel_apply(int n, C *A, int64_t lda, int j, int nbj, int nL, C *backup_col, C *backup_row, int *cert,
              int *counter, int *swapped, int *ipiv, int *info, int *pivoted, PanelPack pk, int no_fallback) {
    panel_apply_cta<C>(n, A, lda, j, nbj, nL, blockIdx.x, gridDim.x, backup_col, backup_row, cert, counter, swapped,
                       ipiv, info, pivoted, pk, no_fallback);
}

// Single-CTA fallback driver when there is no trailing strip (last panel).
template <typename C>
__device__ __forceinline__ void panel_last_cta(int n, C *A, int64_t lda, int j, int nbj, C *backup_col, int *cert,
                                               int *swapped, int *ipiv, int *info, int *pivoted,
                                               int no_fallback = 0) {
    if (no_fallback || *cert == 0) return;
    for (int c = 0; c < nbj; ++c)
        for (int r = threadIdx.x; r < n - j; r += 256) A[(int64_t)(j + c) * lda + j + r] = backup_col[(int64_t)c * n + r];
    __syncthreads();
    pivoted_panel(n, A, lda, j, nbj, ipiv, info, swapped);
    if (threadIdx.x == 0) atomicAdd(pivoted, 1);
}

template <typename C>
__global__ void __launch_bounds__(256)
k_panel_last(int n, C *A, int64_t lda, int j, int nbj, C *backup_col, int *cert, int *swapped, int *ipiv, int *info,
             int *pivoted, int no_fallback) {
    panel_last_cta<C>(n, A, lda, j, nbj, backup_col, cert, swapped, ipiv, info, pivoted, no_fallback);
}

// Apply interchanges of later panels to the columns left of them.
template <typename C>
__device__ __forceinline__ void laswp_left_col(int c, int n, C *A, int64_t lda, int nb, const int *swapped,
                                               const int *ipiv) {
    if (c >= n) return;
    const int npan = (n + nb - 1) / nb;
    C *a = A + (int64_t)c * lda;
    for (int pnl = 0; pnl < npan; ++pnl) {
        const int j = pnl * nb;
        if (!swapped[pnl] || c >= j) continue;
        const int nbj = min(nb, n - j);
        for (int kk = 0; kk < nbj; ++kk) {
            const int p = ipiv[j + kk] - 1;
            if (p != j + kk) {
                const C x = a[j + kk];
                a[j + kk] = a[p];
                a[p] = x;
            }
        }
    }
}

template <typename C>
__global__ void k_laswp_left(int n, C *A, int64_t lda, int nb, const int *swapped, const int *ipiv) {
    laswp_left_col<C>(blockIdx.x * blockDim.x + threadIdx.x, n, A, lda, nb, swapped, ipiv);
}

// ------------------------------------------------------------------ getrs
// ident[0] = 1 when ipiv is the identity permutation (cleared by any entry that is not).
__global__ void k_ipiv_identity(int n, const int *ipiv, int *ident) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && ipiv[i] != i + 1) atomicAnd(ident, 0);
}

template <typename C>
__global__ void k_laswp_rhs(int n, int nrhs, C *B, int64_t ldb, const int *ipiv, const int *ident) {
    if (*ident) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nrhs) return;
    C *b = B + (int64_t)c * ldb;
    for (int i = 0; i < n; ++i) {
        const int p = ipiv[i] - 1;
        if (p != i) {
            const C x = b[i];
            b[i] = b[p];
            b[p] = x;
        }
    }
}

// In-place triangular solve of the nbj-row strip of B at row j with the diagonal block of
// LU at (j, j): UPPER = false -> unit lower L, true -> upper U.  4 lanes per column,
// TRSM_COLS columns per CTA.  Dynamic smem: NB * NBP + NB elements.  Batched over
// blockIdx.y: system y uses LU + y * sLU and B + y * sB.
#define TRSM_COLS 16
template <typename C, bool UPPER>
__global__ void __launch_bounds__(4 * TRSM_COLS)
k_trsm_diag(int nrhs, const C *__restrict__ LU, int64_t lda, C *B, int64_t ldb, int j, int nbj, int64_t sLU,
            int64_t sB) {
    LU += blockIdx.y * sLU;
    B += blockIdx.y * sB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *T = reinterpret_cast<C *>(smem_raw);
    C *rd = T + NB * NBP;
    const int t = threadIdx.x, s = t & 3;
    stage_diag(LU, lda, j, nbj, T, rd);
    const int col = blockIdx.x * TRSM_COLS + (t >> 2);
    const bool ok = col < nrhs;
    C v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int r = 4 * i + s;
        v[i] = (ok && r < nbj) ? B[(int64_t)col * ldb + j + r] : czero<C>();
    }
    if (UPPER) subst_col_upper_loop(v, T, rd, s);
    else subst_col_lower1_loop(v, T, s);
    if (ok) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = 4 * i + s;
            if (r < nbj) B[(int64_t)col * ldb + j + r] = v[i];
        }
    }
}
