// Dense complex LU (getrf), multi-RHS triangular solves (getrs), residuals and
// backward errors on column-major complex128 / complex64 matrices.
//
// Factorization (right-looking, block width NB):
//   for each panel j:
//     k_diag_lu      one CTA: unpivoted LU of the NB x NB diagonal block in shared
//                    memory, inverses of its unit-lower L11 and upper U11, and the
//                    diagonal-pivot certificate inside the block;
//     k_panel_l21    L21 = A21 * inv(U11), backup of the panel, certificate below it;
//     k_panel_fix    one CTA: a no-op unless the certificate failed, in which case it
//                    restores the panel and refactors it with partial pivoting
//                    (argmax by |re|+|im|, first index on ties, as LAPACK izamax);
//     k_row_update   row interchanges of the panel (if any) on the trailing columns,
//                    then U12 = inv(L11) * A12;
//     k_gemm         A22 -= L21 * U12.
// The certificate: partial pivoting chooses the diagonal at step c exactly when
// |a_ic^(c)|_1 <= |a_cc^(c)|_1 for every i > c, and a_ic^(c) = l_ic u_cc, so checking
// |l_ic u_cc|_1 <= |u_cc|_1 over the panel proves that the unpivoted factors are the
// partially pivoted ones (reference linalg/dense.py:114-155, scipy lu_factor/getrf).
#pragma once
#include "common.cuh"

#define LU_NB 64
#define GEMM_BM 64
#define GEMM_BN 64
#define GEMM_BK 16
#define GEMM_THREADS 256

// ------------------------------------------------------------------ generic GEMM
// C[MxN] = (BETA ? C : 0) + (NEG ? -1 : 1) * A[MxK] * B[KxN]; column-major.
template <typename ACC, typename TA, typename TB, typename TC, bool NEG, bool BETA>
__global__ void __launch_bounds__(GEMM_THREADS)
k_gemm(int M, int N, int K, const TA *__restrict__ A, int64_t lda, const TB *__restrict__ B, int64_t ldb,
       TC *__restrict__ C, int64_t ldc) {
    using R = typename real_of<ACC>::type;
    __shared__ ACC As[GEMM_BK][GEMM_BM];
    __shared__ ACC Bs[GEMM_BK][GEMM_BN];
    const int t = threadIdx.x;
    const int tx = t & 15, ty = t >> 4;
    const int m0 = blockIdx.x * GEMM_BM, n0 = blockIdx.y * GEMM_BN;
    ACC acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = czero<ACC>();
    for (int k0 = 0; k0 < K; k0 += GEMM_BK) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = t + GEMM_THREADS * i;
            {
                const int r = e & 63, c = e >> 6;
                const int gm = m0 + r, gk = k0 + c;
                ACC v = czero<ACC>();
                if (gm < M && gk < K) {
                    const TA x = A[(int64_t)gk * lda + gm];
                    v = mk((R)x.x, (R)x.y);
                }
                As[c][r] = v;
            }
            {
                const int r = e & 15, c = e >> 4;
                const int gk = k0 + r, gn = n0 + c;
                ACC v = czero<ACC>();
                if (gk < K && gn < N) {
                    const TB x = B[(int64_t)gn * ldb + gk];
                    v = mk((R)x.x, (R)x.y);
                }
                Bs[r][c] = v;
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GEMM_BK; ++kk) {
            ACC a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) cfma(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + tx + 16 * i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
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

// ------------------------------------------------------------------ triangular inverses
// In shared memory: S holds an nbj x nbj LU block (column-major, leading dim LU_NB).
// Writes inv(L) (unit lower) to Li and inv(U) to Ui (both nbj x nbj, leading dim LU_NB,
// zeros elsewhere).  Row sweeps: inv(U) row i from rows > i, inv(L) row i from rows < i.
template <typename C>
__device__ void tri_inverses(const C *S, int nbj, C *Li, C *Ui) {
    const int t = threadIdx.x, nt = blockDim.x;
    for (int e = t; e < LU_NB * LU_NB; e += nt) {
        Li[e] = czero<C>();
        Ui[e] = czero<C>();
    }
    __syncthreads();
    // inv(L): X[i][c] = delta_ic - sum_{c<=p<i} L[i][p] X[p][c], processed i ascending
    // inv(U): Y[i][c] = (delta_ic - sum_{i<p<=c} U[i][p] Y[p][c]) / U[i][i], i descending
    for (int step = 0; step < nbj; ++step) {
        const int il = step;            // row of inv(L)
        const int iu = nbj - 1 - step;  // row of inv(U)
        for (int c = t; c < 2 * nbj; c += nt) {
            if (c < nbj) {
                if (c <= il) {
                    C acc = (c == il) ? mk((typename real_of<C>::type)1, (typename real_of<C>::type)0) : czero<C>();
                    for (int p = c; p < il; ++p) cfms(acc, S[p * LU_NB + il], Li[c * LU_NB + p]);
                    Li[c * LU_NB + il] = acc;
                }
            } else {
                const int cc = c - nbj;
                if (cc >= iu) {
                    C acc = (cc == iu) ? mk((typename real_of<C>::type)1, (typename real_of<C>::type)0) : czero<C>();
                    for (int p = iu + 1; p <= cc; ++p) cfms(acc, S[p * LU_NB + iu], Ui[cc * LU_NB + p]);
                    Ui[cc * LU_NB + iu] = cdiv(acc, S[iu * LU_NB + iu]);
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ diagonal block
// Dynamic shared memory: 3 * LU_NB * LU_NB elements of C (block, inv L, inv U).
template <typename C>
__global__ void k_diag_lu(int n, C *A, int64_t lda, int j, int nbj, C *linv, C *uinv, C *backup,
                          int *cert, int *ipiv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    C *Li = S + LU_NB * LU_NB;
    C *Ui = Li + LU_NB * LU_NB;
    const int t = threadIdx.x, nt = blockDim.x;
    __shared__ int bad;
    if (t == 0) bad = 0;
    for (int e = t; e < nbj * nbj; e += nt) {
        const int r = e % nbj, c = e / nbj;
        const C v = A[(int64_t)(j + c) * lda + j + r];
        S[c * LU_NB + r] = v;
        backup[(int64_t)c * n + r] = v;  // backup column-major with leading dim n (rows from j)
    }
    for (int r = t; r < nbj; r += nt) ipiv[j + r] = j + r + 1;
    __syncthreads();
    for (int kk = 0; kk < nbj; ++kk) {
        const C piv = S[kk * LU_NB + kk];
        const auto pa = cabs1(piv);
        for (int r = kk + 1 + t; r < nbj; r += nt) {
            const C a = S[kk * LU_NB + r];
            if (!(cabs1(a) <= pa) || pa == 0) bad = 1;
        }
        if (pa == 0 && t == 0) bad = 1;
        __syncthreads();
        if (pa != 0) {
            for (int r = kk + 1 + t; r < nbj; r += nt) S[kk * LU_NB + r] = cdiv(S[kk * LU_NB + r], piv);
        }
        __syncthreads();
        const int rem = nbj - kk - 1;
        for (int e = t; e < rem * rem; e += nt) {
            const int r = kk + 1 + e % rem, c = kk + 1 + e / rem;
            cfms(S[c * LU_NB + r], S[kk * LU_NB + r], S[c * LU_NB + kk]);
        }
        __syncthreads();
    }
    for (int e = t; e < nbj * nbj; e += nt) {
        const int r = e % nbj, c = e / nbj;
        A[(int64_t)(j + c) * lda + j + r] = S[c * LU_NB + r];
    }
    tri_inverses(S, nbj, Li, Ui);
    for (int e = t; e < LU_NB * LU_NB; e += nt) {
        linv[e] = Li[e];
        uinv[e] = Ui[e];
    }
    if (t == 0 && bad) atomicOr(cert, 1);
}

// ------------------------------------------------------------------ L21 = A21 inv(U11)
// Each CTA handles 32 rows below the diagonal block; dynamic smem: 32 x LU_NB elements.
template <typename C>
__global__ void k_panel_l21(int n, C *A, int64_t lda, int j, int nbj, const C *__restrict__ uinv, C *backup,
                            int *cert) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);  // [LU_NB cols][32 rows]
    const int r0 = j + nbj + blockIdx.x * 32;
    const int t = threadIdx.x, nt = blockDim.x;
    const int rows = min(32, n - r0);
    if (rows <= 0) return;
    for (int e = t; e < 32 * nbj; e += nt) {
        const int r = e & 31, c = e >> 5;
        if (r < rows) {
            const C v = A[(int64_t)(j + c) * lda + r0 + r];
            S[c * 32 + r] = v;
            backup[(int64_t)c * n + (r0 - j) + r] = v;
        }
    }
    __syncthreads();
    int bad = 0;
    for (int e = t; e < 32 * nbj; e += nt) {
        const int r = e & 31, c = e >> 5;
        if (r >= rows) continue;
        C acc = czero<C>();
        for (int p = 0; p <= c; ++p) cfma(acc, S[p * 32 + r], uinv[c * LU_NB + p]);
        // certificate: |l u_cc|_1 <= |u_cc|_1 with u_cc from the factored diagonal block
        const C ucc = A[(int64_t)(j + c) * lda + j + c];
        if (!(cabs1(cmul(acc, ucc)) <= cabs1(ucc))) bad = 1;
        A[(int64_t)(j + c) * lda + r0 + r] = acc;
    }
    if (__syncthreads_or(bad) && t == 0) atomicOr(cert, 1);
}

// ------------------------------------------------------------------ pivoted fallback
// One CTA (blockDim multiple of 32, <= 1024). Runs only when *cert != 0.
template <typename C>
__global__ void __launch_bounds__(1024) k_panel_fix(int n, C *A, int64_t lda, int j, int nbj, C *linv, C *uinv, const C *backup,
                            const int *cert, int *swapped, int *ipiv, int *info, int *pivoted_panels) {
    if (*cert == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    C *Li = S + LU_NB * LU_NB;
    C *Ui = Li + LU_NB * LU_NB;
    using R = typename real_of<C>::type;
    __shared__ R wv[32];
    __shared__ int wi[32];
    __shared__ int s_piv;
    __shared__ int s_any;
    const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, warp = t >> 5, nw = nt >> 5;
    const int h = n - j;
    if (t == 0) s_any = 0;
    // restore the panel
    for (int c = 0; c < nbj; ++c)
        for (int r = t; r < h; r += nt) A[(int64_t)(j + c) * lda + j + r] = backup[(int64_t)c * n + r];
    __syncthreads();
    for (int kk = 0; kk < nbj; ++kk) {
        const int col = j + kk;
        R best = (R)-1;
        int bi = 0x7fffffff;
        for (int r = col + t; r < n; r += nt) {
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
        if (warp == 0) {
            best = lane < nw ? wv[lane] : (R)-1;
            bi = lane < nw ? wi[lane] : 0x7fffffff;
            for (int off = 16; off > 0; off >>= 1) {
                const R ov = __shfl_down_sync(0xffffffffu, best, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) {
                s_piv = bi;
                ipiv[col] = bi + 1;
                if (bi != col) s_any = 1;
            }
        }
        __syncthreads();
        const int p = s_piv;
        const C pv = A[(int64_t)col * lda + p];
        const bool zero = (pv.x == 0 && pv.y == 0);
        if (zero) {
            if (t == 0 && *info == 0) *info = col + 1;
        } else if (p != col) {
            for (int c = t; c < nbj; c += nt) {
                C *a = A + (int64_t)(j + c) * lda;
                const C x = a[col];
                a[col] = a[p];
                a[p] = x;
            }
        }
        __syncthreads();
        if (!zero) {
            const C d = A[(int64_t)col * lda + col];
            for (int r = col + 1 + t; r < n; r += nt) A[(int64_t)col * lda + r] = cdiv(A[(int64_t)col * lda + r], d);
        }
        __syncthreads();
        for (int r = col + 1 + t; r < n; r += nt) {
            const C l = A[(int64_t)col * lda + r];
            for (int c = kk + 1; c < nbj; ++c) cfms(A[(int64_t)(j + c) * lda + r], l, A[(int64_t)(j + c) * lda + col]);
        }
        __syncthreads();
    }
    for (int e = t; e < nbj * nbj; e += nt) {
        const int r = e % nbj, c = e / nbj;
        S[c * LU_NB + r] = A[(int64_t)(j + c) * lda + j + r];
    }
    __syncthreads();
    tri_inverses(S, nbj, Li, Ui);
    for (int e = t; e < LU_NB * LU_NB; e += nt) {
        linv[e] = Li[e];
        uinv[e] = Ui[e];
    }
    if (t == 0) {
        *swapped = s_any;
        atomicAdd(pivoted_panels, 1);
    }
}

// ------------------------------------------------------------------ U12 = inv(L11) * P A12
// Each CTA handles 32 trailing columns; dynamic smem: LU_NB x 32 elements.
template <typename C>
__global__ void k_row_update(int n, C *A, int64_t lda, int j, int nbj, const C *__restrict__ linv, const int *swapped,
                             const int *ipiv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);  // [32 cols][LU_NB rows]
    const int c0 = j + nbj + blockIdx.x * 32;
    const int t = threadIdx.x, nt = blockDim.x;
    const int cols = min(32, n - c0);
    if (cols <= 0) return;
    if (*swapped) {
        for (int c = t; c < cols; c += nt) {
            C *a = A + (int64_t)(c0 + c) * lda;
            for (int kk = 0; kk < nbj; ++kk) {
                const int p = ipiv[j + kk] - 1;
                if (p != j + kk) {
                    const C x = a[j + kk];
                    a[j + kk] = a[p];
                    a[p] = x;
                }
            }
        }
        __syncthreads();
    }
    for (int e = t; e < nbj * 32; e += nt) {
        const int r = e % nbj, c = e / nbj;
        if (c < cols) S[c * LU_NB + r] = A[(int64_t)(c0 + c) * lda + j + r];
    }
    __syncthreads();
    for (int e = t; e < nbj * 32; e += nt) {
        const int r = e % nbj, c = e / nbj;
        if (c >= cols) continue;
        C acc = S[c * LU_NB + r];  // unit diagonal
        for (int p = 0; p < r; ++p) cfma(acc, linv[p * LU_NB + r], S[c * LU_NB + p]);
        A[(int64_t)(c0 + c) * lda + j + r] = acc;
    }
}

// Apply interchanges of later panels to the columns left of them.
template <typename C>
__global__ void k_laswp_left(int n, C *A, int64_t lda, int nb, const int *swapped, const int *ipiv) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
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

// ------------------------------------------------------------------ getrs helpers
// All diagonal-block inverses at once: one CTA per block.
template <typename C>
__global__ void k_invert_blocks(int n, const C *LU, int64_t lda, int nb, C *linv_all, C *uinv_all) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    C *Li = S + LU_NB * LU_NB;
    C *Ui = Li + LU_NB * LU_NB;
    const int b = blockIdx.x;
    const int j = b * nb, nbj = min(nb, n - j);
    const int t = threadIdx.x, nt = blockDim.x;
    for (int e = t; e < nbj * nbj; e += nt) {
        const int r = e % nbj, c = e / nbj;
        S[c * LU_NB + r] = LU[(int64_t)(j + c) * lda + j + r];
    }
    __syncthreads();
    tri_inverses(S, nbj, Li, Ui);
    for (int e = t; e < LU_NB * LU_NB; e += nt) {
        linv_all[(int64_t)b * LU_NB * LU_NB + e] = Li[e];
        uinv_all[(int64_t)b * LU_NB * LU_NB + e] = Ui[e];
    }
}

// Row interchanges on the right-hand sides (forward order), one thread per column.
template <typename C>
__global__ void k_laswp_rhs(int n, int nrhs, C *B, int64_t ldb, const int *ipiv) {
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

// X_blk <- T * X_blk in place for the nbj-row strip starting at row j, T = nbj x nbj
// (leading dim LU_NB).  Each CTA handles 32 columns.
template <typename C>
__global__ void k_tri_apply(int nrhs, C *B, int64_t ldb, int j, int nbj, const C *__restrict__ T) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    const int c0 = blockIdx.x * 32;
    const int t = threadIdx.x, nt = blockDim.x;
    const int cols = min(32, nrhs - c0);
    for (int e = t; e < nbj * 32; e += nt) {
        const int r = e % nbj, c = e / nbj;
        if (c < cols) S[c * LU_NB + r] = B[(int64_t)(c0 + c) * ldb + j + r];
    }
    __syncthreads();
    for (int e = t; e < nbj * 32; e += nt) {
        const int r = e % nbj, c = e / nbj;
        if (c >= cols) continue;
        C acc = czero<C>();
        for (int p = 0; p < nbj; ++p) cfma(acc, T[p * LU_NB + r], S[c * LU_NB + p]);
        B[(int64_t)(c0 + c) * ldb + j + r] = acc;
    }
}

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

// Row sums of |A_ij| (modulus): one warp per row-chunk; out[r] = sum_c |A[r, c]|.
template <typename TA>
__global__ void k_row_abs_sum(int n, const TA *__restrict__ A, int64_t lda, double *rowsum) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    double s = 0.0;
    for (int c = 0; c < n; ++c) {
        const TA v = A[(int64_t)c * lda + r];
        s += hypot((double)v.x, (double)v.y);
    }
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
template <typename TX>
__global__ void k_col_absmax3(int m, const double2 *R, int64_t ldr, const TX *X, int64_t ldx, const double2 *B,
                              int64_t ldb, double *out) {
    const int c = blockIdx.x;
    double mr = 0.0, mx = 0.0, mb = 0.0;
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
        const double2 a = R[(int64_t)c * ldr + r];
        const TX x = X[(int64_t)c * ldx + r];
        const double2 b = B[(int64_t)c * ldb + r];
        mr = fmax(mr, hypot(a.x, a.y));
        mx = fmax(mx, hypot((double)x.x, (double)x.y));
        mb = fmax(mb, hypot(b.x, b.y));
    }
    for (int off = 16; off > 0; off >>= 1) {
        mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
        mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, off));
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
            mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
            mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
            mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, off));
        }
        if (lane == 0) { out[3 * c] = mr; out[3 * c + 1] = mx; out[3 * c + 2] = mb; }
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
        if (!(e == e)) e = INFINITY;
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
