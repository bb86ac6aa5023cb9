// Grouped LU: one factorization of many independent systems of different orders (the
// systems of a frequency sweep, the Fourier modes of a body of revolution), advanced in
// lockstep of 64-column panel steps.  Step p runs, for every system still active, the
// same four stages as the single-system factorization (lu.cuh), each as ONE launch over
// all systems:
//   k_grp_diag      one CTA per active system: LU of its diagonal block at column 64 p
//                   (diag_lu_cta, with the diagonal-pivot certificate);
//   k_grp_apply     every 64-row strip of L21 and 64-column strip of U12 of every system
//                   with a trailing matrix (panel_apply_cta; the last CTA of a system runs
//                   that system's pivoted fallback when its certificate failed);
//   k_grp_last      one CTA per system whose last panel this is (panel_last_cta);
//   trailing update A22 -= L21 U12 of every system: complex64 as split-TF32 on tcgen05
//                   (k_grp_apply writes both operands packed, k_grp_tc_update runs
//                   every 128 x 128 output tile of every system, its C tile staged in
//                   shared memory during the main loop), complex128 on the FP64
//                   tensor cores (k_grp_dmma_update, every 64 x 64 tile).
// Systems are ordered by decreasing order, so the systems active at step p are a prefix
// of the list.  A CTA finds its system by binary search in a per-step prefix sum of the
// systems' CTA counts (host-computed once per plan); the per-system pointers are in a
// device table, so that a captured CUDA graph of the whole sequence can be replayed for
// new matrices of the same orders after the table is rewritten.
#pragma once
#include "dmma.cuh"
#include "lu.cuh"
#include "tc_gemm.cuh"

#define GRP_BN 128              // output-tile width of the tensor-core trailing update
#define GRP_STAGES 2              // pipeline stages (4 K-tiles per update; the C tile is staged too)
#define GRP_KP (2 * NB)         // real inner dimension of a complex64 update (K = 64 complex)

struct GrpSys {
    void *A;        // column-major matrix, overwritten by L\U
    int64_t lda;
    int n, npan;
    int *ipiv;      // 1-based pivots (identity unless a panel fell back to partial pivoting)
    void *bcol;     // n x NB backup of the panel columns
    void *brow;     // n x NB backup of the U12 strip
    int *flags;     // [0] info, [1] pivoted panels, cert[npan], swapped[npan], counter[npan]
    float *pa_hi, *pa_lo, *pb_hi, *pb_lo;  // packed L21 / U12 (complex64 systems)
};

// Packed operand rows of a complex64 update with `rest` trailing rows / columns.
__host__ __device__ __forceinline__ int grp_rows_a(int rest) { return (2 * rest + TC_BM - 1) / TC_BM * TC_BM; }
__host__ __device__ __forceinline__ int grp_rows_b(int rest) { return (rest + GRP_BN - 1) / GRP_BN * GRP_BN; }

// Largest s in [0, count) with prefix[s] <= b (prefix strictly increasing, prefix[0] = 0).
__device__ __forceinline__ int grp_find(const int *__restrict__ prefix, int count, int b) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename C>
__global__ void __launch_bounds__(256, 1) k_grp_diag(const GrpSys *__restrict__ sys, int p) {
    const GrpSys &S = sys[blockIdx.x];
    const int j = NB * p, nbj = min(NB, S.n - j);
    diag_lu_cta<C>(S.n, (C *)S.A, S.lda, j, nbj, (C *)S.bcol, S.flags + 2 + p, S.ipiv);
}

// Systems 0..count-1 all have a trailing matrix at step p (rest > 0, so nbj = NB).
template <typename C>
__global__ void __launch_bounds__(256, sizeof(C) == 8 ? 3 : 2) k_grp_apply(const GrpSys *__restrict__ sys, int p, const int *prefix, int count) {
    const int s = grp_find(prefix, count, blockIdx.x);
    const GrpSys &S = sys[s];
    const int j = NB * p, rest = S.n - j - NB, nL = (rest + NB - 1) / NB;
    int *cert = S.flags + 2, *swapped = cert + S.npan, *counter = swapped + S.npan;
    PanelPack pk;  // complex64: the panel solve writes the trailing update's packed operands
    if (sizeof(C) == sizeof(float2)) {
        pk.a_hi = S.pa_hi;
        pk.a_lo = S.pa_lo;
        pk.a_rows = grp_rows_a(rest);
        pk.b_hi = S.pb_hi;
        pk.b_lo = S.pb_lo;
        pk.b_rows = grp_rows_b(rest);
    }
    panel_apply_cta<C>(S.n, (C *)S.A, S.lda, j, NB, nL, blockIdx.x - __ldg(prefix + s), 2 * nL, (C *)S.bcol,
                       (C *)S.brow, cert + p, counter + p, swapped + p, S.ipiv, S.flags, S.flags + 1, pk);
}

// Systems first..first+gridDim.x-1 end at step p.
template <typename C>
__global__ void __launch_bounds__(256) k_grp_last(const GrpSys *__restrict__ sys, int p, int first) {
    const GrpSys &S = sys[first + blockIdx.x];
    const int j = NB * p;
    int *cert = S.flags + 2, *swapped = cert + S.npan;
    panel_last_cta<C>(S.n, (C *)S.A, S.lda, j, S.n - j, (C *)S.bcol, cert + p, swapped + p, S.ipiv, S.flags,
                      S.flags + 1);
}

// Packing of L21 (A operand, grp_rows_a(rest) rows) and U12 (B operand, grp_rows_b(rest)
// rows) of every updating system: rows / 8 CTAs of 256 threads per operand (32 chunks per
// row of GRP_KP floats).
__global__ void __launch_bounds__(256) k_grp_pack(const GrpSys *__restrict__ sys, int p, const int *prefix, int count) {
    const int s = grp_find(prefix, count, blockIdx.x);
    const GrpSys &S = sys[s];
    const int j = NB * p, rest = S.n - j - NB;
    const int Mp = grp_rows_a(rest), Np = grp_rows_b(rest);
    const int b = blockIdx.x - __ldg(prefix + s), ba = Mp / 8;
    const float2 *A = (const float2 *)S.A;
    if (b < ba)
        tc_pack_a_chunk((int64_t)b * 256 + threadIdx.x, rest, NB, A + (int64_t)j * S.lda + j + NB, S.lda, S.pa_hi,
                        S.pa_lo, Mp, Mp, 0, GRP_KP, 1.f);
    else
        tc_pack_b_chunk((int64_t)(b - ba) * 256 + threadIdx.x, NB, rest, A + (int64_t)(j + NB) * S.lda + j, S.lda,
                        S.pb_hi, S.pb_lo, Np, GRP_KP);
}

// A22 -= L21 U12 for every updating complex64 system: (Mp / 128) x (Np / BN) tiles each.
template <int BN, int STAGES>
__global__ void __launch_bounds__(TC_THREADS)
k_grp_tc_update(const GrpSys *__restrict__ sys, int p, const int *prefix, int count, int *err) {
    const int s = grp_find(prefix, count, blockIdx.x);
    const GrpSys &S = sys[s];
    const int j = NB * p, rest = S.n - j - NB;
    const int Mp = grp_rows_a(rest), Np = grp_rows_b(rest), mt = Mp / TC_BM;
    const int t = blockIdx.x - __ldg(prefix + s);
    float2 *A22 = (float2 *)S.A + (int64_t)(j + NB) * S.lda + j + NB;
    tc_gemm_cta<BN, STAGES, true>(GRP_KP / TC_BK, S.pa_hi, S.pa_lo, Mp, S.pb_hi, S.pb_lo, Np, (float *)A22,
                                  2 * S.lda, 2 * rest, rest, -1.f, 0, 0, err, (t % mt) * TC_BM, (t / mt) * BN);
}

// A22 -= L21 U12 for every updating complex128 system: ceil(rest / 64)^2 tiles each.
__global__ void __launch_bounds__(DM_THREADS)
k_grp_dmma_update(const GrpSys *__restrict__ sys, int p, const int *prefix, int count) {
    const int s = grp_find(prefix, count, blockIdx.x);
    const GrpSys &S = sys[s];
    const int j = NB * p, rest = S.n - j - NB, mt = (rest + DM_BM - 1) / DM_BM;
    const int t = blockIdx.x - __ldg(prefix + s);
    const double2 *A = (const double2 *)S.A;
    gemm_dmma_cta<true, true>(rest, rest, NB, A + (int64_t)j * S.lda + j + NB, S.lda, A + (int64_t)(j + NB) * S.lda + j,
                              S.lda, (double2 *)S.A + (int64_t)(j + NB) * S.lda + j + NB, S.lda, (t % mt) * DM_BM,
                              (t / mt) * DM_BN);
}

// Interchanges of later panels applied to the columns left of them; grid (ceil(n_max /
// 128), count).
template <typename C>
__global__ void k_grp_laswp(const GrpSys *__restrict__ sys) {
    const GrpSys &S = sys[blockIdx.y];
    laswp_left_col<C>(blockIdx.x * blockDim.x + threadIdx.x, S.n, (C *)S.A, S.lda, NB, S.flags + 2 + S.npan, S.ipiv);
}

// out[2 i] = info, out[2 i + 1] = pivoted panels of system i.
__global__ void k_grp_flags(const GrpSys *__restrict__ sys, int count, int *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        out[2 * i] = sys[i].flags[0];
        out[2 * i + 1] = sys[i].flags[1];
    }
}
