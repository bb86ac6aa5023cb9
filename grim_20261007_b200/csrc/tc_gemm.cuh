// Complex64 GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32) with FP32-level
// accuracy from a split-TF32 product: x = hi + lo (hi = tf32(x), lo = tf32(x - hi)) and
// A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi, all accumulated in FP32 in tensor memory.
//
// Complex -> real: with C and B viewed as interleaved real column-major matrices
// (C^ is 2M x N, B^ is 2K x N), C^ = A~ B^ where A~ (2M x 2K) expands every complex a into
// the 2 x 2 block [re -im; im re].  No flop is wasted: 2M x N x 2K x 2 = 8 M N K.
//
// Packed operand layout ("tile layout"): a real operand of Rp rows x Kp columns (Rp a
// multiple of the tile height, Kp a multiple of 32) is stored K-tile by K-tile; inside a
// K-tile the Rp rows of 32 floats (128 bytes) follow each other, each row's 16-byte chunk
// c stored at chunk c ^ (r & 7) -- the canonical K-major 128-byte-swizzle order of 8-row,
// 1024-byte atoms.  Rows [r0, r0 + 128) of K-tile kt are therefore one contiguous, already
// swizzled 16 KB block: a single cp.async.bulk moves it into shared memory, where the UMMA
// descriptors read it directly.  Operands are packed once (hi and lo in separate arrays)
// and can be reused by many GEMMs: the blocked triangular solves keep their packed panels
// for every right-hand side of a refinement loop.
//
// Kernel (one 128 x BN output tile per CTA, STAGES-deep pipeline, 128 threads):
//   warp 0, lane 0  producer: waits for a free stage, posts the expected byte count on the
//                   stage's "full" mbarrier and issues 4 bulk copies (A hi/lo, B hi/lo);
//   warp 1, lane 0  MMA issuer: waits for a full stage, issues 3 products x 4 K-steps of
//                   tcgen05.mma (M 128, N BN, K 8) into a BN-column FP32 accumulator in
//                   tensor memory, and commits to the stage's "empty" mbarrier, which frees
//                   the stage for the producer once those MMAs have read it;
//   warps 2-3       meanwhile prefetch this CTA's slice of C into L2;
//   all 4 warps     epilogue after the final commit: tcgen05.ld of the accumulator (warp w
//                   owns TMEM lanes 32w..32w+31 = output rows), then
//                   C = (row in [ow_lo, ow_hi) ? 0 : C) + alpha * D, coalesced along rows.
// Every mbarrier wait is bounded (about one second of clock).  On a timeout the kernel
// records an error flag, stops issuing, waits (bounded) for the copies and MMAs it has in
// flight, frees its tensor memory and returns.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define TC_BM 128
#define TC_BK 32
#define TC_THREADS 128

template <int BN, int STAGES, bool STAGE_C = false>
struct TcCfg {
    static constexpr int A_BYTES = TC_BM * TC_BK * 4;              // one hi or lo A tile
    static constexpr int B_BYTES = BN * TC_BK * 4;                 // one hi or lo B tile
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // Ahi, Alo, Bhi, Blo
    static constexpr int C_BYTES = STAGE_C ? TC_BM * BN * 4 : 0;   // the C tile, staged during the main loop
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + C_BYTES + 1024;
    static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
};

// 8-byte asynchronous global -> shared copy (zero-filled when !valid; src then unused).
__device__ __forceinline__ void cp_async8(uint32_t dst, const void *src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(valid ? 8 : 0) : "memory");
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Float offset of element (r, k) in the tile layout of an operand with Rp rows.
__host__ __device__ __forceinline__ int64_t tc_tile_offset(int r, int k, int Rp) {
    return (int64_t)(k >> 5) * Rp * 32 + (int64_t)r * 32 + ((((k & 31) >> 2) ^ (r & 7)) << 2) + (k & 3);
}

__device__ __forceinline__ void tc_store_chunk(float *hi, float *lo, int64_t off, float v0, float v1, float v2,
                                               float v3) {
    const float h0 = tf32_rna(v0), h1 = tf32_rna(v1), h2 = tf32_rna(v2), h3 = tf32_rna(v3);
    *reinterpret_cast<float4 *>(hi + off) = make_float4(h0, h1, h2, h3);
    *reinterpret_cast<float4 *>(lo + off) =
        make_float4(tf32_rna(v0 - h0), tf32_rna(v1 - h1), tf32_rna(v2 - h2), tf32_rna(v3 - h3));
}

// A~ (2M x 2K real, from complex M x K column-major A) into real rows [r_off, r_off + Mp)
// of an operand with Rp rows in the tile layout, zero padded to Mp x Kp and scaled by
// sign (+1 or -1).  One thread per 16-byte chunk; consecutive threads take consecutive
// rows so that the complex reads are coalesced.
__device__ __forceinline__ void tc_pack_a_chunk(int64_t idx, int M, int K, const float2 *__restrict__ A, int64_t lda,
                                                float *__restrict__ hi, float *__restrict__ lo, int Mp, int Rp,
                                                int r_off, int Kp, float sign) {
    if (idx >= (int64_t)Mp * (Kp >> 2)) return;
    const int r = (int)(idx % Mp), k0 = (int)(idx / Mp) * 4;
    const int m = r >> 1, t = r & 1, kc = k0 >> 1;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (m < M) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (kc + q < K) {
                const float2 a = A[(int64_t)(kc + q) * lda + m];
                v[2 * q] = sign * (t == 0 ? a.x : a.y);
                v[2 * q + 1] = sign * (t == 0 ? -a.y : a.x);
            }
        }
    }
    tc_store_chunk(hi, lo, tc_tile_offset(r_off + r, k0, Rp), v[0], v[1], v[2], v[3]);
}

__global__ void k_tc_pack_a(int M, int K, const float2 *__restrict__ A, int64_t lda, float *__restrict__ hi,
                            float *__restrict__ lo, int Mp, int Rp, int r_off, int Kp, float sign) {
    tc_pack_a_chunk((int64_t)blockIdx.x * blockDim.x + threadIdx.x, M, K, A, lda, hi, lo, Mp, Rp, r_off, Kp, sign);
}

// B^ (rows n < Np, real columns 2k+s = (re, im) of B[k, n]) into the tile layout, zero
// padded.  One thread per 16-byte chunk, consecutive threads along k (coalesced reads and
// writes of a column).
__device__ __forceinline__ void tc_pack_b_chunk(int64_t idx, int K, int N, const float2 *__restrict__ B, int64_t ldb,
                                                float *__restrict__ hi, float *__restrict__ lo, int Np, int Kp) {
    const int kq = Kp >> 2;
    if (idx >= (int64_t)Np * kq) return;
    const int n = (int)(idx / kq), k0 = (int)(idx % kq) * 4, kc = k0 >> 1;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (n < N) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (kc + q < K) {
                const float2 b = B[(int64_t)n * ldb + kc + q];
                v[2 * q] = b.x;
                v[2 * q + 1] = b.y;
            }
        }
    }
    tc_store_chunk(hi, lo, tc_tile_offset(n, k0, Np), v[0], v[1], v[2], v[3]);
}

__global__ void k_tc_pack_b(int K, int N, const float2 *__restrict__ B, int64_t ldb, float *__restrict__ hi,
                            float *__restrict__ lo, int Np, int Kp) {
    tc_pack_b_chunk((int64_t)blockIdx.x * blockDim.x + threadIdx.x, K, N, B, ldb, hi, lo, Np, Kp);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, 128-byte swizzle UMMA shared-memory descriptor: LBO 16 B (ignored), SBO 1024 B.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Bounded wait on an mbarrier phase; false after ~1 s (2e9 clocks).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    for (int i = 0;; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 255) == 255 && clock64() - t0 > 2000000000LL) return false;
    }
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Plain bulk copy global -> this CTA's own shared memory, completing on bar.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// D[tmem] (+)= A[sA] * B[sB]^T for one 32-float K-tile: 4 MMAs of K 8.
__device__ __forceinline__ void umma_ktile_tf32(uint32_t tmem, uint32_t sA, uint32_t sB, uint32_t idesc, bool first) {
#pragma unroll
    for (int kk = 0; kk < TC_BK / 8; ++kk) {
        const uint64_t da = umma_desc_sw128(sA + kk * 32);
        const uint64_t db = umma_desc_sw128(sB + kk * 32);
        const uint32_t acc = (first && kk == 0) ? 0u : 1u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
            :
            : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u)
            : "memory");
    }
}

// C (interleaved complex64 viewed as real, column stride ldc_real floats):
// C[m, n] = (m in [ow_lo, ow_hi) ? 0 : C[m, n]) + alpha * (A~ B^)[m, n]
// for m < Mvalid, n < Nvalid; this CTA computes the tile at rows m0, columns n0.  A and B
// in the tile layout.
//
// STAGE_C: warps 2-3 copy this CTA's C tile into shared memory (8-byte cp.async, one complex
// element per copy) while the main loop runs, and the epilogue reads it from there, so no
// global load waits in the epilogue; without it they only prefetch the tile into L2.
template <int BN, int STAGES, bool STAGE_C = false>
__device__ __forceinline__ void tc_gemm_cta(int nk, const float *__restrict__ Ahi, const float *__restrict__ Alo,
                                            int Mp, const float *__restrict__ Bhi, const float *__restrict__ Blo,
                                            int Np, float *__restrict__ C, int64_t ldc_real, int Mvalid, int Nvalid,
                                            float alpha, int ow_lo, int ow_hi, int *err, int m0, int n0) {
    using Cfg = TcCfg<BN, STAGES, STAGE_C>;
    extern __shared__ __align__(1024) unsigned char smem_dyn[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;
    const uint32_t base = (smem_addr(smem_dyn) + 1023u) & ~1023u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_addr(&full[s]), 1);
            mbar_init(smem_addr(&empty[s]), 1);
        }
        mbar_init(smem_addr(&done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    volatile int *vfail = &s_fail;

    if (warp == 0) {
        if (lane == 0) {
            // producer
            int issued = 0;
            for (int kt = 0; kt < nk; ++kt) {
                const int s = kt % STAGES;
                if (kt >= STAGES && !mbar_wait(smem_addr(&empty[s]), ((kt / STAGES) + 1) & 1)) {
                    *vfail = 1;
                    break;
                }
                if (*vfail) break;
                const uint32_t sA = base + s * Cfg::STAGE_BYTES, sAl = sA + Cfg::A_BYTES, sB = sAl + Cfg::A_BYTES,
                               sBl = sB + Cfg::B_BYTES;
                const uint32_t fb = smem_addr(&full[s]);
                mbar_expect_tx(fb, Cfg::STAGE_BYTES);
                const int64_t aoff = (int64_t)kt * Mp * 32 + (int64_t)m0 * 32;
                const int64_t boff = (int64_t)kt * Np * 32 + (int64_t)n0 * 32;
                bulk_g2s(sA, Ahi + aoff, Cfg::A_BYTES, fb);
                bulk_g2s(sAl, Alo + aoff, Cfg::A_BYTES, fb);
                bulk_g2s(sB, Bhi + boff, Cfg::B_BYTES, fb);
                bulk_g2s(sBl, Blo + boff, Cfg::B_BYTES, fb);
                issued = kt + 1;
            }
            // on the failure path, copies issued but not yet consumed must land before exit
            if (*vfail) {
                for (int kt = (issued > STAGES ? issued - STAGES : 0); kt < issued; ++kt)
                    mbar_wait(smem_addr(&full[kt % STAGES]), (kt / STAGES) & 1);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(TC_BM >> 4) << 24);
            for (int kt = 0; kt < nk; ++kt) {
                const int s = kt % STAGES;
                if (!mbar_wait(smem_addr(&full[s]), (kt / STAGES) & 1)) {
                    *vfail = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t sA = base + s * Cfg::STAGE_BYTES, sAl = sA + Cfg::A_BYTES, sB = sAl + Cfg::A_BYTES,
                               sBl = sB + Cfg::B_BYTES;
                umma_ktile_tf32(tmem, sA, sB, idesc, kt == 0);
                umma_ktile_tf32(tmem, sA, sBl, idesc, false);
                umma_ktile_tf32(tmem, sAl, sB, idesc, false);
                umma_commit(smem_addr(&empty[s]));
            }
            umma_commit(smem_addr(&done));  // arrives once every MMA issued above has completed
        }
        __syncwarp();
    } else if (STAGE_C) {
        // warps 2-3: C tile -> shared memory, [column][128 rows] floats; thread t copies the
        // complex element (real rows 2t, 2t+1) of every column (zero outside the matrix and
        // in the overwrite window)
        const int t = threadIdx.x - 64, r = m0 + 2 * t;
        const bool row_ok = r < Mvalid && !(r >= ow_lo && r < ow_hi);
        const uint32_t sC = base + STAGES * Cfg::STAGE_BYTES + 8 * t;
        for (int c = 0; c < BN; ++c) {
            const bool ok = row_ok && n0 + c < Nvalid;
            cp_async8(sC + c * (TC_BM * 4), ok ? (const void *)(C + (int64_t)(n0 + c) * ldc_real + r) : (const void *)C,
                      ok);
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
    } else {
        // warps 2-3: pull this CTA's slice of C into L2 while the main loop runs
        // (one 128-byte line per prefetch; rows of the overwrite window are not read)
        const int lines_per_col = TC_BM / 32;
        for (int e = threadIdx.x - 64; e < BN * lines_per_col; e += 64) {
            const int n = n0 + e / lines_per_col, r = m0 + (e % lines_per_col) * 32;
            if (n < Nvalid && r < Mvalid && !(r >= ow_lo && r + 32 <= ow_hi))
                asm volatile("prefetch.global.L2 [%0];" ::"l"(C + (int64_t)n * ldc_real + r));
        }
    }
    // everyone: wait for the accumulator (bounded)
    if (!mbar_wait(smem_addr(&done), 0)) *vfail = 1;
    __syncthreads();
    if (*vfail) {
        if (threadIdx.x == 0) atomicOr(err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int m = m0 + warp * 32 + lane;
        const bool row_ok = m < Mvalid, ow = m >= ow_lo && m < ow_hi;
#pragma unroll 1
        for (int c = 0; c < BN; c += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row_ok) {
                // all 16 loads first, then the stores (no load waits behind a store)
                float cv[16];
                if (STAGE_C) {
                    const float *sCf = reinterpret_cast<const float *>(smem_dyn + (base - smem_addr(smem_dyn)) +
                                                                       STAGES * Cfg::STAGE_BYTES);
#pragma unroll
                    for (int j = 0; j < 16; ++j) cv[j] = sCf[(c + j) * TC_BM + (m - m0)];
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int n = n0 + c + j;
                        cv[j] = (!ow && n < Nvalid) ? C[(int64_t)n * ldc_real + m] : 0.f;
                    }
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c + j;
                    if (n < Nvalid) C[(int64_t)n * ldc_real + m] = cv[j] + alpha * __uint_as_float(v[j]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
    }
}

// grid = (Mp / 128, Np / BN).
template <int BN, int STAGES, bool STAGE_C = false>
__global__ void __launch_bounds__(TC_THREADS)
k_tc_gemm(int nk, const float *__restrict__ Ahi, const float *__restrict__ Alo, int Mp, const float *__restrict__ Bhi,
          const float *__restrict__ Blo, int Np, float *__restrict__ C, int64_t ldc_real, int Mvalid, int Nvalid,
          float alpha, int ow_lo, int ow_hi, int *err) {
    tc_gemm_cta<BN, STAGES, STAGE_C>(nk, Ahi, Alo, Mp, Bhi, Blo, Np, C, ldc_real, Mvalid, Nvalid, alpha, ow_lo, ow_hi,
                                     err, blockIdx.x * TC_BM, blockIdx.y * BN);
}
