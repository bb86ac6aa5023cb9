// Partial-pivoting panel factorization on a thread-block cluster (LAPACK getf2 order, the
// reference's scipy lu_factor pivots: |re| + |im|, first row on ties).
//
// The 64-column panel rows j..n-1 are spread over the CS CTAs of one cluster, CTA c holding
// panel rows [c rpc, (c+1) rpc) in shared memory (rows past its capacity in a global
// scratch, which stays in L2).  Column step k:
//   1. every CTA finds its best candidate for column k among its rows >= k, and publishes
//      the candidate's whole row (and row k, if it owns it) in a double-buffered slot;
//   2. one cluster barrier;
//   3. every CTA reads the CS candidates through distributed shared memory, takes the
//      largest (first row on ties), copies the winning row p, and the owners of rows k
//      and p swap them (from the published copies);
//   4. l = a_rk / a_kk and a_rc -= l a_kc on the CTA's own rows.
// One cluster barrier per column: a slot is rewritten two steps later, after every CTA
// has passed the barrier that follows its reads.  Every CTA runs the same steps, barriers
// included, whatever its rows.
//
// The panel's interchanges reach the other columns in two ways: the trailing columns take
// them before U12 is formed (k_panel_u_moves, from a list of at most 128 row moves that
// CTA 0 derives from the 64 interchanges), the factored columns on the left at the end of
// the factorization (k_laswp_left, from ipiv).
#pragma once
#include <cooperative_groups.h>

#include "lu.cuh"

namespace cg = cooperative_groups;

#define GEPP_THREADS 256
#define GEPP_LDR (NB + 1)   // padded row stride of the panel rows in shared memory
#define GEPP_MAX_MOVES (2 * NB)

template <typename C>
struct GeppPub {
    C row[NB];    // the CTA's best candidate row of this step
    C krow[NB];   // panel row k, from the CTA that owns it
    double val;   // |re| + |im| of the candidate in column k (-1: no row >= k)
    int idx;      // its panel row
    int pad;
};

// Fixed shared memory of the panel kernel (the rows follow it).
template <typename C>
__host__ __device__ constexpr size_t gepp_fixed_smem() {
    return (2 * sizeof(GeppPub<C>) + NB * sizeof(C) /* prow */ + (size_t)GEPP_THREADS / 32 * 16 /* reduce */ +
            4 * NB * sizeof(int) /* ipiv, first, slot, content */ + 2 * NB * sizeof(int) /* extras */ + 64 + 15) /
           16 * 16;
}

// Better candidate: larger |re| + |im|, then the smaller row.
__device__ __forceinline__ bool gepp_better(double v, int i, double bv, int bi) {
    return v > bv || (v == bv && i < bi);
}

template <typename C>
__global__ void __launch_bounds__(GEPP_THREADS)
k_panel_gepp(int n, C *__restrict__ A, int64_t lda, int j, int nbj, int rpc, int rows_smem, C *__restrict__ gscratch,
             int *__restrict__ ipiv, int *__restrict__ info, int *__restrict__ swapped, int *__restrict__ moves,
             PanelPack pk) {
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    extern __shared__ __align__(16) unsigned char gepp_smem[];
    GeppPub<C> *pub = reinterpret_cast<GeppPub<C> *>(gepp_smem);
    C *prow = reinterpret_cast<C *>(pub + 2);
    double *red_v = reinterpret_cast<double *>(prow + NB);
    int *red_i = reinterpret_cast<int *>(red_v + GEPP_THREADS / 32);
    int *ipiv_s = red_i + GEPP_THREADS / 32;
    int *first = ipiv_s + NB, *slot = first + NB, *content = slot + NB, *extra = content + 2 * NB;
    C *rows = reinterpret_cast<C *>(gepp_smem + gepp_fixed_smem<C>());
    __shared__ int s_p, s_w, s_zero, s_nextra;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m = n - j;
    const int r0 = rank * rpc;
    const int nr = max(0, min(m - r0, rpc));
    C *gs = gscratch + (size_t)rank * (size_t)max(0, rpc - rows_smem) * NB;
    auto rowp = [&](int r) -> C * { return r < rows_smem ? rows + (size_t)r * GEPP_LDR : gs + (size_t)(r - rows_smem) * NB; };

    // load the CTA's rows (coalesced along each column)
    for (int e = tid; e < nr * NB; e += GEPP_THREADS) {
        const int c = e / nr, r = e - c * nr;
        rowp(r)[c] = c < nbj ? A[(int64_t)(j + c) * lda + j + r0 + r] : czero<C>();
    }
    __syncthreads();

    for (int k = 0; k < nbj; ++k) {
        const int par = k & 1;
        // 1. local candidate for column k among rows >= k
        double bv = -1.0;
        int bi = 0x7fffffff;
        for (int r = tid; r < nr; r += GEPP_THREADS) {
            const int g = r0 + r;
            if (g >= k) {
                const double v = (double)cabs1(rowp(r)[k]);
                if (gepp_better(v, g, bv, bi)) { bv = v; bi = g; }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (gepp_better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < GEPP_THREADS / 32; ++w)
                if (gepp_better(red_v[w], red_i[w], bv, bi)) { bv = red_v[w]; bi = red_i[w]; }
            pub[par].val = bv;
            pub[par].idx = bi;
            red_i[0] = bi;
        }
        __syncthreads();
        const int best = red_i[0];
        if (tid < NB) {
            if (best != 0x7fffffff) pub[par].row[tid] = rowp(best - r0)[tid];
            if (k >= r0 && k < r0 + nr) pub[par].krow[tid] = rowp(k - r0)[tid];
        }
        // 2. every CTA's candidate is published
        cluster.sync();
        // 3. the winner: largest |re| + |im|, first row on ties
        if (warp == 0) {
            double v = -1.0;
            int i = 0x7fffffff, w = 0;
            if (lane < (int)cluster.num_blocks()) {
                const GeppPub<C> *rp = cluster.map_shared_rank(&pub[par], lane);
                v = rp->val;
                i = rp->idx;
                w = lane;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, v, o);
                const int oi = __shfl_down_sync(0xffffffffu, i, o);
                const int ow = __shfl_down_sync(0xffffffffu, w, o);
                if (gepp_better(ov, oi, v, i)) { v = ov; i = oi; w = ow; }
            }
            if (lane == 0) {
                s_p = i;
                s_w = w;
                s_zero = !(v > 0.0);
                if (rank == 0) ipiv_s[k] = i;
            }
        }
        __syncthreads();
        const int p = s_p;
        const bool zero = s_zero;
        const int ck = k / rpc, cp = p / rpc;
        if (tid < NB) {
            const C pv = cluster.map_shared_rank(&pub[par], s_w)->row[tid];
            prow[tid] = pv;
            if (p != k && !zero) {
                if (rank == ck) rowp(k - r0)[tid] = pv;
                if (rank == cp) rowp(p - r0)[tid] = cluster.map_shared_rank(&pub[par], ck)->krow[tid];
            }
        }
        __syncthreads();
        if (zero) {
            // LAPACK getf2: a zero pivot column is left as it is, info records its first
            if (rank == 0 && tid == 0) atomicCAS(info, 0, j + k + 1);
            continue;
        }
        // 4. multipliers, then the rank-1 update of the CTA's rows below k
        const C rp = crecip(prow[k]);
        for (int r = tid; r < nr; r += GEPP_THREADS) {
            if (r0 + r > k) {
                C *a = rowp(r);
                a[k] = cmul(a[k], rp);
            }
        }
        __syncthreads();
        const int c = tid & (NB - 1), rg = tid >> 6;
        if (c > k) {
            const C u = prow[c];
            for (int r = rg; r < nr; r += GEPP_THREADS / NB) {
                if (r0 + r > k) {
                    C *a = rowp(r);
                    cfms(a[c], a[k], u);
                }
            }
        }
        __syncthreads();
    }
    // every CTA has finished reading every other CTA's slots before any CTA exits
    cluster.sync();

    // write the factored rows back; complex64: the trailing update's packed A operand (L21)
    for (int e = tid; e < nr * NB; e += GEPP_THREADS) {
        const int cc = e / nr, r = e - cc * nr;
        if (cc < nbj) A[(int64_t)(j + cc) * lda + j + r0 + r] = rowp(r)[cc];
    }
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (pk.a_hi) {
            // L21 rows are panel rows >= nbj (= NB here); padding rows up to a_rows / 2 are zero
            const int rest = m - nbj;
            const int pad_rows = pk.a_rows / 2;
            for (int e = tid; e < rpc * NB; e += GEPP_THREADS) {
                const int cc = e / rpc, r = e - cc * rpc;
                const int mrow = r0 + r - nbj;
                if (mrow < 0 || mrow >= pad_rows) continue;
                float xr = 0.f, xi = 0.f;
                if (mrow < rest && r < nr) {
                    const float2 x = *reinterpret_cast<const float2 *>(&rowp(r)[cc]);
                    xr = x.x;
                    xi = x.y;
                }
                pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow, 2 * cc, pk.a_rows), xr, -xi);
                pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow + 1, 2 * cc, pk.a_rows), xi, xr);
            }
            // rows past the rows of every CTA (rpc * CS may not reach pad_rows): zero
            const int covered = (int)cluster.num_blocks() * rpc - nbj;
            if (rank == 0)
                for (int e = tid; e < (pad_rows - covered) * NB; e += GEPP_THREADS) {
                    const int mrow = covered + e / NB, cc = e % NB;
                    if (mrow < 0) continue;
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow, 2 * cc, pk.a_rows), 0.f, 0.f);
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow + 1, 2 * cc, pk.a_rows), 0.f, 0.f);
                }
        }
    }

    // CTA 0: ipiv, the swapped flag and the row moves of the panel's interchanges
    if (rank != 0) return;
    if (tid < nbj) ipiv[j + tid] = j + ipiv_s[tid] + 1;
    if (warp == 0) {
        // first[k]: the first interchange with the same target row; extra targets (rows >= nbj)
        // get slots nbj, nbj + 1, ... in order of first appearance
        for (int k = lane; k < nbj; k += 32) {
            int f = k;
            for (int q = 0; q < k; ++q)
                if (ipiv_s[q] == ipiv_s[k]) { f = q; break; }
            first[k] = f;
        }
        __syncwarp();
        int base = 0;
        for (int k0 = 0; k0 < nbj; k0 += 32) {
            const int k = k0 + lane;
            const bool is_new = k < nbj && ipiv_s[k] >= nbj && first[k] == k;
            const unsigned bal = __ballot_sync(0xffffffffu, is_new);
            if (is_new) {
                const int at = base + __popc(bal & ((1u << lane) - 1u));
                slot[k] = nbj + at;
                extra[at] = ipiv_s[k];
            }
            base += __popc(bal);
        }
        __syncwarp();
        if (lane == 0) {
            s_nextra = base;
            // simulate the interchanges on the touched rows: content[s] = original row now at slot s
            for (int s = 0; s < nbj + base; ++s) content[s] = s < nbj ? s : extra[s - nbj];
            int any = 0;
            for (int k = 0; k < nbj; ++k) {
                const int pk_ = ipiv_s[k];
                if (pk_ == k) continue;
                any = 1;
                const int sp = pk_ < nbj ? pk_ : slot[first[k]];
                const int t = content[k];
                content[k] = content[sp];
                content[sp] = t;
            }
            *swapped = any;
            int cnt = 0;
            for (int s = 0; s < nbj + base; ++s) {
                const int pos = s < nbj ? s : extra[s - nbj];
                if (content[s] != pos) {
                    moves[1 + cnt] = j + pos;                        // destination row
                    moves[1 + GEPP_MAX_MOVES + cnt] = j + content[s];  // source row
                    ++cnt;
                }
            }
            moves[0] = cnt;
        }
    }
}

// U12 = inv(L11) A12 of the trailing columns after the panel's row moves: one CTA per 64
// columns, 4 threads per column.  Each column gathers every move's source before writing
// any destination.  complex64: also writes the trailing update's packed B operand.
// Dynamic smem: NB * NBP + NB elements (the diagonal block and its reciprocals).
template <typename C>
__global__ void __launch_bounds__(256)
k_panel_u_moves(int n, C *__restrict__ A, int64_t lda, int j, int nbj, const int *__restrict__ moves, PanelPack pk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *T = reinterpret_cast<C *>(smem_raw);
    C *rd = T + NB * NBP;
    __shared__ int s_dst[GEPP_MAX_MOVES], s_src[GEPP_MAX_MOVES];
    __shared__ int s_cnt;
    const int t = threadIdx.x, s = t & 3, lane_vec = t >> 2;
    if (t == 0) s_cnt = min(moves[0], GEPP_MAX_MOVES);
    __syncthreads();
    const int cnt = s_cnt;
    for (int i = t; i < cnt; i += 256) {
        s_dst[i] = moves[1 + i];
        s_src[i] = moves[1 + GEPP_MAX_MOVES + i];
    }
    __syncthreads();
    const int col = j + nbj + NB * blockIdx.x + lane_vec;
    const bool ok = col < n;
    // every source of the column is read (by its 4 threads, one warp) before any destination
    // is written; the warp barriers stay outside the per-column condition, which differs
    // between the lanes of a warp at the matrix edge
    C *a = A + (int64_t)col * lda;
    C tmp[GEPP_MAX_MOVES / 4];
    if (ok) {
#pragma unroll
        for (int q = 0; q < GEPP_MAX_MOVES / 4; ++q) {
            const int i = 4 * q + s;
            if (i < cnt) tmp[q] = a[s_src[i]];
        }
    }
    __syncwarp();
    if (ok) {
#pragma unroll
        for (int q = 0; q < GEPP_MAX_MOVES / 4; ++q) {
            const int i = 4 * q + s;
            if (i < cnt) a[s_dst[i]] = tmp[q];
        }
    }
    __syncwarp();
    stage_diag(A, lda, j, nbj, T, rd);
    C v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int r = 4 * i + s;
        v[i] = (ok && r < nbj) ? A[(int64_t)col * lda + j + r] : czero<C>();
    }
    subst_col_lower1(v, T, nbj, s);
    if (ok) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = 4 * i + s;
            if (r < nbj) A[(int64_t)col * lda + j + r] = v[i];
        }
    }
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (pk.b_hi) {
            const int nb_row = NB * blockIdx.x + lane_vec;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int r = 4 * i + s;
                pack_pair(pk.b_hi, pk.b_lo, tc_tile_offset(nb_row, 2 * r, pk.b_rows), ok ? (float)v[i].x : 0.f,
                          ok ? (float)v[i].y : 0.f);
            }
        }
    }
}
