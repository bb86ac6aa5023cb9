// Complex64 GEMM update C -= A B on the 5th-generation tensor cores (tcgen05, kind::tf32),
// with FP32-level accuracy from a split-TF32 product: x = hi + lo (hi = tf32(x),
// lo = tf32(x - hi)) and A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi, all accumulated in FP32
// in tensor memory.
//
// Complex -> real: with C and B viewed as interleaved real column-major matrices
// (C^ is 2M x N, B^ is 2K x N), C^ = A~ B^ where A~ (2M x 2K) expands every complex a into
// the 2 x 2 block [re -im; im re].  The operands are packed once into K-major row-major
// float arrays (k_tc_pack_a: A~ rows of length 2K; k_tc_pack_b: B^ columns of length 2K),
// split into hi and lo, zero padded to the tile grid.
//
// Tile: 128 real rows (64 complex rows) x 64 columns, K in stages of 32 floats (one
// 128-byte row).  Shared-memory tiles use the canonical K-major 128-byte-swizzle layout
// (8-row atoms of 1024 B, 16-byte chunk c of row r at chunk c ^ (r & 7)), filled with
// cp.async by all 128 threads, two stages.  Thread 0 issues the tcgen05.mma
// instructions (4 K-steps x 3 products per stage) into a 64-column FP32 accumulator in
// tensor memory and commits them to the stage's mbarrier; all four warps then read the
// accumulator with tcgen05.ld (warp w owns lanes 32w..32w+31 = rows) and apply C -= D.
// Every mbarrier wait is bounded (about one second of clock); on timeout the kernel
// records an error flag, stops issuing, frees its tensor memory and returns.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define TC_BM 128
#define TC_BN 64
#define TC_BK 32
#define TC_THREADS 128
#define TC_STAGE_BYTES (2 * TC_BM * TC_BK * 4 + 2 * TC_BN * TC_BK * 4)  // Ahi, Alo, Bhi, Blo
#define TC_SMEM_BYTES (2 * TC_STAGE_BYTES + 1024)

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// A~ packing: hi/lo[r * Kp + c] for r < Mp (real rows), c < Kp (real K), zero padded.
__global__ void k_tc_pack_a(int M, int K, const float2 *__restrict__ A, int64_t lda, float *__restrict__ hi,
                            float *__restrict__ lo, int Mp, int Kp) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)Mp * Kp) return;
    const int r = (int)(idx / Kp), c = (int)(idx % Kp);
    const int m = r >> 1, t = r & 1, k = c >> 1, s = c & 1;
    float v = 0.f;
    if (m < M && k < K) {
        const float2 a = A[(int64_t)k * lda + m];
        v = t == 0 ? (s == 0 ? a.x : -a.y) : (s == 0 ? a.y : a.x);
    }
    const float h = tf32_rna(v);
    hi[idx] = h;
    lo[idx] = tf32_rna(v - h);
}

// B^ packing: hi/lo[n * Kp + c] = (re, im) of B[c >> 1, n], n < Np, zero padded.
__global__ void k_tc_pack_b(int K, int N, const float2 *__restrict__ B, int64_t ldb, float *__restrict__ hi,
                            float *__restrict__ lo, int Np, int Kp) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)Np * Kp) return;
    const int n = (int)(idx / Kp), c = (int)(idx % Kp);
    const int k = c >> 1, s = c & 1;
    float v = 0.f;
    if (n < N && k < K) {
        const float2 b = B[(int64_t)n * ldb + k];
        v = s == 0 ? b.x : b.y;
    }
    const float h = tf32_rna(v);
    hi[idx] = h;
    lo[idx] = tf32_rna(v - h);
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

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

// Load one stage: rows [row0, row0 + rows) of a packed array (row length Kp floats),
// columns [k0, k0 + 32), into a swizzled tile at smem address tile.
__device__ __forceinline__ void tc_load_tile(uint32_t tile, const float *__restrict__ src, int row0, int rows,
                                             int Kp, int k0) {
    for (int e = threadIdx.x; e < rows * 8; e += TC_THREADS) {
        const int r = e >> 3, c = e & 7;
        const uint32_t dst = tile + (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
        cp_async16(dst, src + (int64_t)(row0 + r) * Kp + k0 + 4 * c);
    }
}

// C (interleaved complex64 viewed as real, column stride ldc_real floats) -= D.
// grid = (Mp / 128, Np / 64).  Mvalid real rows and N columns are written.
__global__ void __launch_bounds__(TC_THREADS)
k_tc_gemm_sub(int Kp, const float *__restrict__ Ahi, const float *__restrict__ Alo, const float *__restrict__ Bhi,
              const float *__restrict__ Blo, float *__restrict__ C, int64_t ldc_real, int Mvalid, int N, int *err) {
    extern __shared__ __align__(1024) unsigned char smem_dyn[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;
    // 1024-aligned stage bases inside the dynamic allocation
    const uint32_t base = (smem_addr(smem_dyn) + 1023u) & ~1023u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * TC_BN;
    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int s = 0; s < 2; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(TC_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                           ((uint32_t)(TC_BM >> 4) << 24);
    const int nk = Kp / TC_BK;
    uint32_t uses[2] = {0u, 0u};
    bool ok = true;
    for (int kt = 0; kt < nk && ok; ++kt) {
        const int st = kt & 1;
        if (kt >= 2) {
            if (!mbar_wait(smem_addr(&bar[st]), (uses[st] - 1) & 1)) ok = false;
        }
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        const uint32_t sA = base + st * TC_STAGE_BYTES;
        const uint32_t sAl = sA + TC_BM * TC_BK * 4;
        const uint32_t sB = sAl + TC_BM * TC_BK * 4;
        const uint32_t sBl = sB + TC_BN * TC_BK * 4;
        tc_load_tile(sA, Ahi, m0, TC_BM, Kp, kt * TC_BK);
        tc_load_tile(sAl, Alo, m0, TC_BM, Kp, kt * TC_BK);
        tc_load_tile(sB, Bhi, n0, TC_BN, Kp, kt * TC_BK);
        tc_load_tile(sBl, Blo, n0, TC_BN, Kp, kt * TC_BK);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t pa[3] = {sA, sA, sAl}, pb[3] = {sB, sBl, sB};
#pragma unroll
            for (int pr = 0; pr < 3; ++pr) {
#pragma unroll
                for (int kk = 0; kk < TC_BK / 8; ++kk) {
                    const uint64_t da = umma_desc_sw128(pa[pr] + kk * 32);
                    const uint64_t db = umma_desc_sw128(pb[pr] + kk * 32);
                    const uint32_t acc = (kt > 0 || pr > 0 || kk > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                        :
                        : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&bar[st]))
                         : "memory");
        }
        uses[st]++;
    }
    // wait for the last commit (it tracks every MMA issued before it)
    if (ok && nk > 0) {
        const int st = (nk - 1) & 1;
        if (!mbar_wait(smem_addr(&bar[st]), (uses[st] - 1) & 1)) ok = false;
    }
    if (!ok) s_fail = 1;
    __syncthreads();
    if (s_fail) {
        if (threadIdx.x == 0) atomicOr(err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int m = m0 + warp * 32 + lane;
#pragma unroll
        for (int c = 0; c < TC_BN; c += 8) {
            uint32_t v[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < Mvalid) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int n = n0 + c + j;
                    if (n < N) C[(int64_t)n * ldc_real + m] -= __uint_as_float(v[j]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN) : "memory");
    }
}
