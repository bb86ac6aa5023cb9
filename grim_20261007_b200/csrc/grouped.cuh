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
    int static_pivot;  // 1: no partial-pivoting fallback (the caller guards the solution)
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
                       (C *)S.brow, cert + p, counter + p, swapped + p, S.ipiv, S.flags, S.flags + 1, pk,
                       S.static_pivot);
}

// Systems first..first+gridDim.x-1 end at step p.
template <typename C>
__global__ void __launch_bounds__(256) k_grp_last(const GrpSys *__restrict__ sys, int p, int first) {
    const GrpSys &S = sys[first + blockIdx.x];
    const int j = NB * p;
    int *cert = S.flags + 2, *swapped = cert + S.npan;
    panel_last_cta<C>(S.n, (C *)S.A, S.lda, j, S.n - j, (C *)S.bcol, cert + p, swapped + p, S.ipiv, S.flags,
                      S.flags + 1, S.static_pivot);
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

// Persistent form of k_grp_tc_update: one CTA per SM walks the step's tiles (t = blockIdx.x,
// blockIdx.x + gridDim.x, ...), so that one tile's epilogue overlaps the next tile's operand
// loads and MMAs and the set-up (barriers, tensor memory) is paid once per SM.  192 threads:
//   warp 0 (lane 0)  producer: bulk copies of the packed operands into a 2-stage ring;
//   warp 1 (lane 0)  MMA issuer: 3 split-TF32 products per K-tile into one of two BN-column
//                    accumulators (tile i uses accumulator i & 1), commit per stage and per tile;
//   warps 2-5        epilogue: each thread owns one output row (TMEM lane quadrant = warp % 4),
//                    copies its row of the C tile into shared memory (4-byte cp.async) while the
//                    tile's MMAs run, then C = C + alpha D and releases the accumulator.
// Every wait is bounded; on a timeout the CTA records the error flag, stops, waits (bounded) for
// its copies and MMAs in flight, frees its tensor memory and returns.
#define GRP_P_THREADS 192

// BN 128: 2 stages of 64 KB + a 64 KB C tile; BN 64: 4 stages of 48 KB + a 32 KB C tile.
template <int BN>
struct GrpPCfg {
    static constexpr int STAGES = BN == 128 ? 2 : 4;
    static constexpr int A_BYTES = TC_BM * TC_BK * 4;
    static constexpr int B_BYTES = BN * TC_BK * 4;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int C_BYTES = TC_BM * BN * 4;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + C_BYTES + 1024;
    static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(valid ? 4 : 0) : "memory");
}

// Tile t of step p: its system and the tile's origin (real rows m0, columns n0).
struct GrpTile {
    const GrpSys *S;
    int rest, Mp, Np, m0, n0;
};

template <int BN>
__device__ __forceinline__ GrpTile grp_tile(const GrpSys *__restrict__ sys, int p, const int *prefix, int count,
                                            int t) {
    GrpTile g;
    const int s = grp_find(prefix, count, t);
    g.S = &sys[s];
    g.rest = g.S->n - NB * p - NB;
    g.Mp = grp_rows_a(g.rest);
    g.Np = grp_rows_b(g.rest);
    const int mt = g.Mp / TC_BM, local = t - __ldg(prefix + s);
    g.m0 = (local % mt) * TC_BM;
    g.n0 = (local / mt) * BN;
    return g;
}

template <int BN>
__global__ void __launch_bounds__(GRP_P_THREADS, 1)
k_grp_tc_update_p(const GrpSys *__restrict__ sys, int p, const int *prefix, int count, int ntiles, int *err) {
    using Cfg = GrpPCfg<BN>;
    constexpr int NK = GRP_KP / TC_BK;
    extern __shared__ __align__(1024) unsigned char smem_dyn[];
    __shared__ __align__(8) uint64_t full[Cfg::STAGES], empty[Cfg::STAGES], tfull[2], tempty[2], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;
    const uint32_t base = (smem_addr(smem_dyn) + 1023u) & ~1023u;
    const uint32_t sC = base + Cfg::STAGES * Cfg::STAGE_BYTES;
    float *sCf = reinterpret_cast<float *>(smem_dyn + (base - smem_addr(smem_dyn)) + Cfg::STAGES * Cfg::STAGE_BYTES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int i = 0; i < Cfg::STAGES; ++i) {
            mbar_init(smem_addr(&full[i]), 1);
            mbar_init(smem_addr(&empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(smem_addr(&tfull[i]), 1);
            mbar_init(smem_addr(&tempty[i]), 4);  // one arrival per epilogue warp
        }
        mbar_init(smem_addr(&done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(2 * BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    volatile int *vfail = &s_fail;
    const int j = NB * p;

    if (warp == 0) {
        if (lane == 0) {
            int g = 0, issued = 0;
            for (int t = blockIdx.x; t < ntiles && !*vfail; t += gridDim.x) {
                const GrpTile tl = grp_tile<BN>(sys, p, prefix, count, t);
                for (int kt = 0; kt < NK; ++kt, ++g) {
                    const int st = g % Cfg::STAGES;
                    if (g >= Cfg::STAGES &&
                        !mbar_wait(smem_addr(&empty[st]), ((g / Cfg::STAGES) + 1) & 1)) {
                        *vfail = 1;
                        break;
                    }
                    const uint32_t sA = base + st * Cfg::STAGE_BYTES, sAl = sA + Cfg::A_BYTES,
                                   sB = sAl + Cfg::A_BYTES, sBl = sB + Cfg::B_BYTES;
                    const uint32_t fb = smem_addr(&full[st]);
                    mbar_expect_tx(fb, Cfg::STAGE_BYTES);
                    const int64_t aoff = (int64_t)kt * tl.Mp * 32 + (int64_t)tl.m0 * 32;
                    const int64_t boff = (int64_t)kt * tl.Np * 32 + (int64_t)tl.n0 * 32;
                    bulk_g2s(sA, tl.S->pa_hi + aoff, Cfg::A_BYTES, fb);
                    bulk_g2s(sAl, tl.S->pa_lo + aoff, Cfg::A_BYTES, fb);
                    bulk_g2s(sB, tl.S->pb_hi + boff, Cfg::B_BYTES, fb);
                    bulk_g2s(sBl, tl.S->pb_lo + boff, Cfg::B_BYTES, fb);
                    issued = g + 1;
                }
            }
            if (*vfail) {  // copies issued but not consumed must land before the CTA exits
                for (int q = (issued > Cfg::STAGES ? issued - Cfg::STAGES : 0); q < issued; ++q)
                    mbar_wait(smem_addr(&full[q % Cfg::STAGES]), (q / Cfg::STAGES) & 1);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(TC_BM >> 4) << 24);
            int g = 0, i = 0;
            for (int t = blockIdx.x; t < ntiles && !*vfail; t += gridDim.x, ++i) {
                const int acc = i & 1;
                if (i >= 2 && !mbar_wait(smem_addr(&tempty[acc]), ((i / 2) + 1) & 1)) {
                    *vfail = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(acc * BN);
                bool ok = true;
                for (int kt = 0; kt < NK; ++kt, ++g) {
                    const int st = g % Cfg::STAGES;
                    if (!mbar_wait(smem_addr(&full[st]), (g / Cfg::STAGES) & 1)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sA = base + st * Cfg::STAGE_BYTES, sAl = sA + Cfg::A_BYTES,
                                   sB = sAl + Cfg::A_BYTES, sBl = sB + Cfg::B_BYTES;
                    umma_ktile_tf32(d, sA, sB, idesc, kt == 0);
                    umma_ktile_tf32(d, sA, sBl, idesc, false);
                    umma_ktile_tf32(d, sAl, sB, idesc, false);
                    umma_commit(smem_addr(&empty[st]));
                }
                if (!ok) {
                    *vfail = 1;
                    break;
                }
                umma_commit(smem_addr(&tfull[acc]));
            }
            umma_commit(smem_addr(&done));  // arrives once every MMA issued above has completed
        }
        __syncwarp();
    } else {
        // epilogue warps 2-5: TMEM lane quadrant q = warp % 4 holds output rows 32 q .. 32 q + 31
        const int q = warp & 3, row = 32 * q + lane;
        const uint32_t sRow = sC + 4 * row;
        int i = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
            if (*vfail) break;
            const GrpTile tl = grp_tile<BN>(sys, p, prefix, count, t);
            float *C = (float *)tl.S->A + 2 * ((int64_t)(j + NB) * tl.S->lda + j + NB);
            const int64_t ldc = 2 * tl.S->lda;
            const int Mvalid = 2 * tl.rest, Nvalid = tl.rest, m = tl.m0 + row;
            const bool row_ok = m < Mvalid;
            for (int c = 0; c < BN; ++c) {  // this thread's row of C (only it reads it back)
                const bool ok = row_ok && tl.n0 + c < Nvalid;
                cp_async4(sRow + c * (TC_BM * 4), ok ? (const void *)(C + (int64_t)(tl.n0 + c) * ldc + m)
                                                     : (const void *)C,
                          ok);
            }
            asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
            const int acc = i & 1;
            if (!mbar_wait(smem_addr(&tfull[acc]), (i / 2) & 1)) {
                *vfail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                uint32_t v[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * BN + c)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (row_ok) {
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const int n = tl.n0 + c + jj;
                        if (n < Nvalid)
                            C[(int64_t)n * ldc + m] = sCf[(c + jj) * TC_BM + row] - __uint_as_float(v[jj]);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&tempty[acc]));
        }
    }
    // every MMA has completed before the tensor memory is released (bounded)
    if (!mbar_wait(smem_addr(&done), 0)) *vfail = 1;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*vfail && threadIdx.x == 0) atomicOr(err, 1);
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN) : "memory");
    }
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
