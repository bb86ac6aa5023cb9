// Complex128 GEMM C = (BETA ? C : 0) + (NEG ? -1 : 1) A B on the FP64 tensor cores
// (mma.sync m8n8k4 .f64, the only FP64 tensor-core instruction; tcgen05 has no FP64 kind).
//
// CTA tile 64 x 64 complex, 4 warps in 2 x 2, each warp 32 x 32 complex = 4 x 4 MMA tiles
// with separate real and imaginary FP64 accumulators (64 doubles per thread).  One
// complex k-step of a tile is four real MMAs:
//   re += Ar Br,  re += (-Ai) Bi,  im += Ar Bi,  im += Ai Br.
// K in stages of 8 complex (two MMA k-steps), three shared-memory stages filled with
// cp.async (16 bytes = one complex element, zero-filled outside the matrices).
// Fragments of m8n8k4 (PTX ISA): A 8 x 4 row-major, lane holds A[lane / 4][lane % 4];
// B 4 x 8 column-major, lane holds B[lane % 4][lane / 4]; C 8 x 8, lane holds
// C[lane / 4][2 (lane % 4) + {0, 1}].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DM_BM 64
#define DM_BN 64
#define DM_BK 8
#define DM_STAGES 3
#define DM_THREADS 128
#define DM_LDA (DM_BM + 2)  // padded leading dims of the shared tiles (complex elements)
#define DM_LDB (DM_BN + 2)
#define DM_SMEM_BYTES (DM_STAGES * DM_BK * (DM_LDA + DM_LDB) * 16)

__device__ __forceinline__ void dm_cp16(void *smem, const void *gmem, bool valid) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    const int bytes = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gmem), "r"(bytes) : "memory");
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool NEG, bool BETA>
__device__ __forceinline__ void gemm_dmma_cta(int M, int N, int K, const double2 *__restrict__ A, int64_t lda,
                                              const double2 *__restrict__ B, int64_t ldb, double2 *__restrict__ C,
                                              int64_t ldc, int m0, int n0) {
    extern __shared__ __align__(16) unsigned char dm_smem[];
    double2 *As = reinterpret_cast<double2 *>(dm_smem);               // [stage][k][DM_LDA]
    double2 *Bs = As + DM_STAGES * DM_BK * DM_LDA;                     // [stage][k][DM_LDB] (k-major rows of n)
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int g = lane >> 2, q = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int nk = (K + DM_BK - 1) / DM_BK;

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kt * DM_BK;
        double2 *as = As + stage * DM_BK * DM_LDA;
        double2 *bs = Bs + stage * DM_BK * DM_LDB;
#pragma unroll
        for (int i = 0; i < (DM_BM * DM_BK) / DM_THREADS; ++i) {
            const int e = t + DM_THREADS * i;
            const int m = e % DM_BM, k = e / DM_BM;  // consecutive threads: consecutive rows of a column
            const int gm = m0 + m, gk = k0 + k;
            const bool ok = gm < M && gk < K;
            dm_cp16(as + k * DM_LDA + m, ok ? (const void *)(A + (int64_t)gk * lda + gm) : (const void *)A, ok);
        }
#pragma unroll
        for (int i = 0; i < (DM_BN * DM_BK) / DM_THREADS; ++i) {
            const int e = t + DM_THREADS * i;
            const int k = e % DM_BK, n = e / DM_BK;  // consecutive threads: consecutive k of a column of B
            const int gk = k0 + k, gn = n0 + n;
            const bool ok = gk < K && gn < N;
            dm_cp16(bs + k * DM_LDB + n, ok ? (const void *)(B + (int64_t)gn * ldb + gk) : (const void *)B, ok);
        }
    };

    double re[4][4][2], im[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) re[i][j][0] = re[i][j][1] = im[i][j][0] = im[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < DM_STAGES - 1; ++s) {
        if (s < nk) load_stage(s, s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kt = 0; kt < nk; ++kt) {
        asm volatile("cp.async.wait_group %0;" ::"n"(DM_STAGES - 2) : "memory");
        __syncthreads();
        // prefetch stage kt + STAGES - 1 into the buffer freed by stage kt - 1
        if (kt + DM_STAGES - 1 < nk) load_stage((kt + DM_STAGES - 1) % DM_STAGES, kt + DM_STAGES - 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        const double2 *as = As + (kt % DM_STAGES) * DM_BK * DM_LDA;
        const double2 *bs = Bs + (kt % DM_STAGES) * DM_BK * DM_LDB;
#pragma unroll
        for (int ks = 0; ks < DM_BK; ks += 4) {
            double ar[4], ai[4], nai[4], br[4], bi[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double2 a = as[(ks + q) * DM_LDA + wm + 8 * i + g];
                ar[i] = a.x;
                ai[i] = a.y;
                nai[i] = -a.y;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double2 b = bs[(ks + q) * DM_LDB + wn + 8 * j + g];
                br[j] = b.x;
                bi[j] = b.y;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    dmma(re[i][j][0], re[i][j][1], ar[i], br[j]);
                    dmma(re[i][j][0], re[i][j][1], nai[i], bi[j]);
                    dmma(im[i][j][0], im[i][j][1], ar[i], bi[j]);
                    dmma(im[i][j][0], im[i][j][1], ai[i], br[j]);
                }
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // epilogue: lane holds rows wm + 8 i + g, columns wn + 8 j + 2 q + {0, 1}
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + wm + 8 * i + g;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int gn = n0 + wn + 8 * j + 2 * q + c;
                if (gn >= N) continue;
                double vr = re[i][j][c], vi = im[i][j][c];
                if (NEG) {
                    vr = -vr;
                    vi = -vi;
                }
                double2 *p = C + (int64_t)gn * ldc + gm;
                if (BETA) {
                    const double2 o = *p;
                    vr += o.x;
                    vi += o.y;
                }
                *p = make_double2(vr, vi);
            }
        }
    }
}

// grid = (ceil(M / 64), ceil(N / 64)).
template <bool NEG, bool BETA>
__global__ void __launch_bounds__(DM_THREADS)
k_gemm_dmma(int M, int N, int K, const double2 *__restrict__ A, int64_t lda, const double2 *__restrict__ B,
            int64_t ldb, double2 *__restrict__ C, int64_t ldc) {
    gemm_dmma_cta<NEG, BETA>(M, N, K, A, lda, B, ldb, C, ldc, blockIdx.x * DM_BM, blockIdx.y * DM_BN);
}
