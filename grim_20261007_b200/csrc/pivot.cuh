// Partial-pivoting panel factorization on a thread-block cluster (LAPACK getf2 order, the
// reference's scipy lu_factor pivots: |re| + |im|, first row on ties).
//
// The 64-column panel rows j..n-1 are spread over the CS CTAs of one cluster, CTA c holding
// panel rows [c rpc, (c+1) rpc) in shared memory (rows past its capacity in a global
// scratch, which stays in L2).  Column step k:
//   1. every CTA reduces its best candidate for column k among its rows >= k, pushes its
//      (value, row) into every CTA's shared memory and publishes the candidate's whole row
//      (and row k, if it owns it) in a double-buffered slot, with step k - 1's rank-1
//      update (still pending on columns > k) applied on the fly;
//   2. it arrives at the cluster barrier, finishes that pending update on its own rows
//      while the other CTAs arrive, and waits;
//   3. one warp finds the winner among the pushed candidates, then reads its row and row
//      k through distributed shared memory; the owners of rows k and p swap them;
//   4. one thread per row forms l = a_rk / a_kk, updates column k + 1 at once and finds
//      the candidates of step k + 1.
// One cluster barrier per column: a slot (pushed or published) is rewritten two steps
// later, after every CTA has passed the barrier that follows its reads.  Every CTA runs the same steps, barriers
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
    return (2 * sizeof(GeppPub<C>) + 2 * NB * sizeof(C) /* prow */ + (size_t)GEPP_THREADS / 32 * 16 /* reduce */ +
            4 * NB * sizeof(int) /* ipiv, first, slot, content */ + 2 * NB * sizeof(int) /* extras */ + 64 + 15) /
           16 * 16;
}

// Better candidate: larger |re| + |im|, then the smaller row.
__device__ __forceinline__ bool gepp_better(double v, int i, double bv, int bi) {
    return v > bv || (v == bv && i < bi);
}

// Row moves of one panel's interchanges (one warp): ipiv_s[k] is the panel row that step k
// swapped with row k (k < nbj).  Simulating the swaps on the touched rows -- the panel's
// first nbj rows and the targets below them -- gives, for each touched row, the row whose
// content ends there: moves[0] = count, then count destination rows and, GEPP_MAX_MOVES
// entries on, count source rows (absolute: + j).  Scratch (shared): first, slot (NB ints),
// content (2 NB), extra (NB).  Returns the count (every lane).
__device__ __forceinline__ int panel_moves(const int *ipiv_s, int nbj, int j, int *moves, int *first, int *slot,
                                           int *content, int *extra) {
    const int lane = threadIdx.x & 31;
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
    int cnt = 0;
    if (lane == 0) {
        for (int s = 0; s < nbj + base; ++s) content[s] = s < nbj ? s : extra[s - nbj];
        for (int k = 0; k < nbj; ++k) {
            const int pk_ = ipiv_s[k];
            if (pk_ == k) continue;
            const int sp = pk_ < nbj ? pk_ : slot[first[k]];
            const int t = content[k];
            content[k] = content[sp];
            content[sp] = t;
        }
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
    return __shfl_sync(0xffffffffu, cnt, 0);
}

// Row moves of every panel of a factorization, from its ipiv (1-based, absolute): one warp
// per panel, moves of panel p at moves_all + p * GEPP_MOVES_STRIDE.
#define GEPP_MOVES_STRIDE (1 + 2 * GEPP_MAX_MOVES)
__global__ void __launch_bounds__(128) k_ipiv_moves(int n, const int *__restrict__ ipiv, int *__restrict__ moves_all) {
    __shared__ int sc[4][NB * 6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * 4 + warp;
    const int npan = (n + NB - 1) / NB;
    if (p >= npan) return;
    const int j = p * NB, nbj = min(NB, n - j);
    int *ip = sc[warp], *first = ip + NB, *slot = first + NB, *content = slot + NB, *extra = content + 2 * NB;
    for (int k = lane; k < nbj; k += 32) ip[k] = ipiv[j + k] - 1 - j;
    __syncwarp();
    panel_moves(ip, nbj, j, moves_all + (size_t)p * GEPP_MOVES_STRIDE, first, slot, content, extra);
}

// Applies the row moves of panels first.. npan-1 to columns of B (one CTA per column, the
// rows it can change staged in shared memory): the interchanges of getrs' right-hand
// sides (left = 0: every panel, every row) and of the factored columns left of later
// panels (left = 1: column c of panel c / NB takes the panels after it, rows from the next
// panel on).  ident (may be NULL): nothing to do when *ident is set.  Dynamic smem: n
// elements (n * sizeof(C) <= GEPP_MOVES_SMEM_MAX).
#define GEPP_MOVES_SMEM_MAX (200 * 1024)
template <typename C>
__global__ void __launch_bounds__(256)
k_apply_moves(int n, C *__restrict__ B, int64_t ldb, int col0, int left, const int *__restrict__ moves_all,
              const int *__restrict__ ident) {
    extern __shared__ __align__(16) unsigned char mv_smem[];
    C *col = reinterpret_cast<C *>(mv_smem);
    const int c = col0 + blockIdx.x;
    const int npan = (n + NB - 1) / NB;
    const int first = left ? c / NB + 1 : 0;
    if (first >= npan || (ident && *ident)) return;
    const int row0 = first * NB;
    C *b = B + (int64_t)c * ldb;
    for (int r = row0 + threadIdx.x; r < n; r += blockDim.x) col[r - row0] = b[r];
    __syncthreads();
    for (int p = first; p < npan; ++p) {
        const int *mv = moves_all + (size_t)p * GEPP_MOVES_STRIDE;
        const int cnt = min(mv[0], GEPP_MAX_MOVES);
        C v = czero<C>();
        const bool act = threadIdx.x < cnt;
        if (act) v = col[mv[1 + GEPP_MAX_MOVES + threadIdx.x] - row0];
        __syncthreads();
        if (act) col[mv[1 + threadIdx.x] - row0] = v;
        __syncthreads();
    }
    for (int r = row0 + threadIdx.x; r < n; r += blockDim.x) b[r] = col[r - row0];
}

// A CTA's candidate of one step, pushed into every CTA of the cluster.
struct GeppCand {
    double val;
    int idx;
    int pad;
};

// Cluster barrier halves: the arrive of threads whose writes other CTAs read carries release
// semantics, the others' is relaxed; the wait acquires.
__device__ __forceinline__ void gepp_arrive(bool release) {
    if (release) asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    else asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void gepp_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

template <typename C>
__global__ void __launch_bounds__(GEPP_THREADS)
k_panel_gepp(int n, C *__restrict__ A, int64_t lda, int j, int nbj, int rpc, int rows_smem, C *__restrict__ gscratch,
             int *__restrict__ ipiv, int *__restrict__ info, int *__restrict__ swapped, int *__restrict__ moves,
             PanelPack pk) {
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int cs = (int)cluster.num_blocks();
    extern __shared__ __align__(16) unsigned char gepp_smem[];
    GeppPub<C> *pub = reinterpret_cast<GeppPub<C> *>(gepp_smem);
    C *prow = reinterpret_cast<C *>(pub + 2);  // [2][NB]: the pivot rows of the last two steps
    double *red_v = reinterpret_cast<double *>(prow + 2 * NB);
    int *red_i = reinterpret_cast<int *>(red_v + GEPP_THREADS / 32);
    int *ipiv_s = red_i + GEPP_THREADS / 32;
    int *first = ipiv_s + NB, *slot = first + NB, *content = slot + NB, *extra = content + 2 * NB;
    C *rows = reinterpret_cast<C *>(gepp_smem + gepp_fixed_smem<C>());
    __shared__ GeppCand cand[2][16];  // [parity][rank]: every CTA's candidate, pushed here
    __shared__ int s_p, s_zero;
    __shared__ C s_rp;

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

    // Step k starts with column k up to date on every row g >= k and the rank-1 update of
    // step k - 1 still pending on columns > k (multipliers in column k - 1, pivot row in
    // prow[(k - 1) & 1]); it finishes it while the cluster barrier completes.
    double bv = -1.0;
    int bi = 0x7fffffff;
    for (int r = tid; r < nr; r += GEPP_THREADS) {
        const double v = (double)cabs1(rowp(r)[0]);
        if (gepp_better(v, r0 + r, bv, bi)) { bv = v; bi = r0 + r; }
    }
    for (int k = 0; k < nbj; ++k) {
        const int par = k & 1;
        const C *uprev = prow + (par ^ 1) * NB;
        // 1. the CTA's candidate for column k: warp maxima, then every thread takes the
        //    largest of the 8 (first row on ties)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (gepp_better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
        __syncthreads();
        bv = red_v[0];
        bi = red_i[0];
#pragma unroll
        for (int w = 1; w < GEPP_THREADS / 32; ++w)
            if (gepp_better(red_v[w], red_i[w], bv, bi)) { bv = red_v[w]; bi = red_i[w]; }
        //    published with the pending update applied: its row (threads 0-63), row k if this
        //    CTA owns it (64-127); its (value, row) pushed into every CTA (warp 4)
        if (tid < 2 * NB) {
            const int c = tid & (NB - 1);
            const int src = tid < NB ? bi : k;
            const bool want = tid < NB ? bi != 0x7fffffff : (k >= r0 && k < r0 + nr);
            if (want) {
                const C *a = rowp(src - r0);
                C x = a[c];
                if (k > 0 && c > k) cfms(x, a[k - 1], uprev[c]);
                if (tid < NB) pub[par].row[c] = x;
                else pub[par].krow[c] = x;
            }
        } else if (warp == 4 && lane < cs) {
            GeppCand *dst = cluster.map_shared_rank(&cand[par][rank], lane);
            dst->val = bv;
            dst->idx = bi;
        }
        // the published rows are read before any warp applies the pending update to them
        __syncthreads();
        gepp_arrive(warp <= 4);
        // 2. the pending update of step k - 1 on the CTA's rows >= k, columns > k: two
        //    threads per row, alternate columns
        if (k > 0) {
            const int half = tid & 1;
            for (int r = tid >> 1; r < nr; r += GEPP_THREADS / 2) {
                if (r0 + r >= k) {
                    C *a = rowp(r);
                    const C l = a[k - 1];
#pragma unroll 4
                    for (int c = k + 1 + half; c < NB; c += 2) cfms(a[c], l, uprev[c]);
                }
            }
        }
        gepp_wait();
        __syncthreads();
        // 3. warp 0: the winner from the pushed candidates (local), then its row and row k
        //    through distributed shared memory; the owners of rows k and p swap them
        if (warp == 0) {
            double v = -1.0;
            int i = 0x7fffffff;
            for (int w = 0; w < cs; ++w) {
                const GeppCand cw = cand[par][w];
                if (gepp_better(cw.val, cw.idx, v, i)) { v = cw.val; i = cw.idx; }
            }
            const bool zero = !(v > 0.0);
            const int ck = k / rpc, cw = i == 0x7fffffff ? 0 : i / rpc;
            const GeppPub<C> *wp = cluster.map_shared_rank(&pub[par], cw);
            const GeppPub<C> *kp = cluster.map_shared_rank(&pub[par], ck);
            const C x0 = wp->row[lane], x1 = wp->row[lane + 32];
            const C k0 = kp->krow[lane], k1 = kp->krow[lane + 32];
            prow[par * NB + lane] = x0;
            prow[par * NB + lane + 32] = x1;
            if (lane == (k & 31)) s_rp = zero ? one_c<C>() : crecip(k < 32 ? x0 : x1);
            if (i != k && !zero) {
                if (rank == ck) {
                    C *a = rowp(k - r0);
                    a[lane] = x0;
                    a[lane + 32] = x1;
                }
                if (rank == cw) {
                    C *a = rowp(i - r0);
                    a[lane] = k0;
                    a[lane + 32] = k1;
                }
            }
            if (lane == 0) {
                s_p = i;
                s_zero = zero;
                if (rank == 0) ipiv_s[k] = zero ? k : i;
            }
        }
        __syncthreads();
        const bool zero = s_zero;
        if (zero && rank == 0 && tid == 0) atomicCAS(info, 0, j + k + 1);
        // 4. multipliers of the CTA's rows below k (LAPACK leaves a zero pivot column
        //    unscaled), column k + 1 updated at once, and the candidates of step k + 1
        const C *u = prow + par * NB;
        const C rp = s_rp;
        bv = -1.0;
        bi = 0x7fffffff;
        for (int r = tid; r < nr; r += GEPP_THREADS) {
            const int g = r0 + r;
            if (g > k) {
                C *a = rowp(r);
                const C l = zero ? a[k] : cmul(a[k], rp);
                a[k] = l;
                if (k + 1 < NB) {
                    cfms(a[k + 1], l, u[k + 1]);
                    const double v = (double)cabs1(a[k + 1]);
                    if (gepp_better(v, g, bv, bi)) { bv = v; bi = g; }
                }
            }
        }
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
        const int cnt = panel_moves(ipiv_s, nbj, j, moves, first, slot, content, extra);
        if (lane == 0) *swapped = cnt > 0;
    }
}

// ------------------------------------------------------------ register-resident panel rows
// The same column steps with every panel row in registers: two threads per row, the thread
// of parity h holding columns h, h + 2, ..., h + 62.  The rank-1 updates then run from
// registers and only pivot rows pass through shared memory.  Each CTA holds at most
// GEPPR_ROWS rows, so the kernel takes panels of at most 16 x GEPPR_ROWS rows.  The
// column steps are instantiated one by one (gepp_reg_step<K>), so every register index is a
// compile-time constant.
//
// Candidates are compared as integer keys: the bits of |re| + |im| (a non-negative double)
// plus one order like the values, 0 marks "no candidate" (and NaN, which LAPACK's search
// never picks either).  Rows rise with the lane, the warp and the CTA, so the lowest holder
// of the maximum key is LAPACK's first row on ties.  Per step, a CTA publishes its best
// row and row k as they are in registers, with the row's multiplier of the previous step;
// the CTAs that read a row apply that pending update to the columns they take.  The
// candidate is pushed with its element in column k, so the winner's reciprocal is formed
// while its row is in flight, and every CTA but the owner of row k fetches only the
// columns right of k.
#define GEPPR_ROWS (GEPP_THREADS / 2)

template <typename C>
struct GeppPushed {
    C piv;                   // the candidate's element in column k
    unsigned long long key;  // its key (0: the CTA has no row >= k)
    int idx;                 // its panel row
    int pad;
};

template <typename C>
struct GeppRegShared {
    C row[2][NB];   // [parity]: the CTA's best candidate row, as in registers
    C krow[2][NB];  // [parity]: panel row k, from the CTA that owns it
    C row_l[2];     // [parity]: their multipliers of the previous step
    C krow_l[2];
    C u[2][NB];     // [parity]: the pivot row of the step (local copy, columns > k)
    C kin[NB];      // row k, in the CTA that owns the winner row
    GeppPushed<C> cand[2][16];  // [parity][rank]: every CTA's candidate, pushed here
    unsigned long long red_k[GEPP_THREADS / 32];
    int red_l[GEPP_THREADS / 32];
    int ipiv[NB], first[NB], slot[NB], content[2 * NB], extra[NB];
    int p, zero;
    C rp;
};

template <typename C>
struct GeppRegThread {
    C a[NB / 2];             // a[q]: column 2 q + half of the thread's row
    C lp;                    // the row's multiplier of the previous step
    unsigned long long key;  // candidate key for the current column (thread holding it)
};

struct GeppRegCtx {
    int tid, lane, warp, half, pr, r0, rank, cs, rpc, nbj, j;
    bool valid;
    int *info;
};

__device__ __forceinline__ unsigned long long gepp_key(double v) {
    return v == v ? (unsigned long long)__double_as_longlong(v) + 1ull : 0ull;
}

// Warp maximum of the keys (every lane) and the lowest lane that holds it (-1: all zero).
__device__ __forceinline__ int gepp_warp_argmax(unsigned long long key, unsigned long long &kmax) {
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    kmax = ((unsigned long long)mhi << 32) | mlo;
    const unsigned bal = __ballot_sync(0xffffffffu, kmax != 0ull && key == kmax);
    return bal ? __ffs(bal) - 1 : -1;
}

template <typename C, int K>
__device__ __forceinline__ void gepp_reg_step(GeppRegThread<C> &st, GeppRegShared<C> &sh, const GeppRegCtx &cx) {
    if (K >= cx.nbj) return;
    cg::cluster_group cluster = cg::this_cluster();
    constexpr int par = K & 1, hk = K & 1, qk = K >> 1;
    const C *uprev = sh.u[par ^ 1];

    // 1. the CTA's candidate for column K: the first warp holding the maximum key
    unsigned long long wmax;
    const int wl = gepp_warp_argmax(st.key, wmax);
    if (cx.lane == 0) {
        sh.red_k[cx.warp] = wmax;
        sh.red_l[cx.warp] = wl;
    }
    __syncthreads();
    unsigned long long cmax = sh.red_k[0];
    int cwarp = 0;
#pragma unroll
    for (int w = 1; w < GEPP_THREADS / 32; ++w)
        if (sh.red_k[w] > cmax) {
            cmax = sh.red_k[w];
            cwarp = w;
        }
    const int owner = cmax ? cwarp * 32 + sh.red_l[cwarp] : 0;  // thread holding the element
    const int bi = cmax ? cx.r0 + (owner >> 1) : 0x7fffffff;
    //    its row and row K published as they are, with their pending multipliers
    const bool own_best = cx.valid && cx.pr == bi;
    const bool own_k = cx.valid && cx.pr == K;
    if (own_best || own_k) {
#pragma unroll
        for (int q = 0; q < NB / 2; ++q) {
            const int c = 2 * q + cx.half;
            if (own_best) sh.row[par][c] = st.a[q];
            if (own_k) sh.krow[par][c] = st.a[q];
        }
        if (cx.half == 0) {
            if (own_best) sh.row_l[par] = st.lp;
            if (own_k) sh.krow_l[par] = st.lp;
        }
    }
    //    (key, row, element) pushed into every CTA by the lanes of the owner's warp
    const int pw = owner >> 5;
    if (cx.warp == pw) {
        const C piv = shfl_c(st.a[qk], owner & 31);
        if (cx.lane < cx.cs) {
            GeppPushed<C> pc;
            pc.piv = piv;
            pc.key = cmax;
            pc.idx = bi;
            pc.pad = 0;
            *cluster.map_shared_rank(&sh.cand[par][cx.rank], cx.lane) = pc;
        }
    }
    const int kw = (K >= cx.r0 && K < cx.r0 + cx.rpc) ? (2 * (K - cx.r0)) >> 5 : -1;
    __syncwarp();
    gepp_arrive(cx.warp == pw || cx.warp == kw);

    // 2. the pending update of step K - 1 on the thread's row (rows >= K, columns > K)
    if (K > 0 && cx.valid && cx.pr >= K) {
#pragma unroll
        for (int q = 0; q < NB / 2; ++q) {
            const int c = 2 * q + cx.half;
            if (c > K) cfms(st.a[q], st.lp, uprev[c]);
        }
    }
    __syncwarp();
    gepp_wait();

    // 3. warp 0: the winner among the pushed candidates (the first CTA holding the maximum),
    //    its columns > K (all of them in the CTA that owns row K), and row K in the CTA that
    //    owns the winner, through distributed shared memory
    if (cx.warp == 0) {
        unsigned long long gmax;
        const int wlane = gepp_warp_argmax(cx.lane < cx.cs ? sh.cand[par][cx.lane].key : 0ull, gmax);
        const bool zero = gmax <= 1ull;  // every candidate 0 (or none finite): no interchange
        const int i = wlane >= 0 ? sh.cand[par][wlane].idx : K;
        const int ck = K / cx.rpc, cw = i / cx.rpc;
        const bool in_ck = cx.rank == ck;
        const C *wrow = wlane >= 0 ? cluster.map_shared_rank(&sh.row[par][0], cw)
                                   : cluster.map_shared_rank(&sh.krow[par][0], ck);
        const C *wlp = wlane >= 0 ? cluster.map_shared_rank(&sh.row_l[par], cw)
                                  : cluster.map_shared_rank(&sh.krow_l[par], ck);
        const int c0 = cx.lane, c1 = cx.lane + 32;
        C x0 = czero<C>(), x1 = czero<C>();
        if (in_ck || c0 > K) x0 = wrow[c0];
        if (in_ck || c1 > K) x1 = wrow[c1];
        const bool need_k = cx.rank == cw && i != K && !zero;
        C k0 = czero<C>(), k1 = czero<C>(), kl = czero<C>();
        if (need_k) {
            const C *kr = cluster.map_shared_rank(&sh.krow[par][0], ck);
            k0 = kr[c0];
            k1 = kr[c1];
            kl = *cluster.map_shared_rank(&sh.krow_l[par], ck);
        }
        if (cx.lane == 0) {
            sh.rp = zero ? one_c<C>() : crecip(sh.cand[par][wlane].piv);
            sh.p = i;
            sh.zero = zero;
            if (cx.rank == 0) sh.ipiv[K] = zero ? K : i;
        }
        if (K > 0) {
            const C wl_ = *wlp;
            if (c0 > K) cfms(x0, wl_, uprev[c0]);
            if (c1 > K) cfms(x1, wl_, uprev[c1]);
            if (need_k) {
                if (c0 > K) cfms(k0, kl, uprev[c0]);
                if (c1 > K) cfms(k1, kl, uprev[c1]);
            }
        }
        sh.u[par][c0] = x0;
        sh.u[par][c1] = x1;
        if (need_k) {
            sh.kin[c0] = k0;
            sh.kin[c1] = k1;
        }
    }
    __syncthreads();

    // 4. rows K and p swap; multipliers of the rows below K (LAPACK leaves a zero pivot
    //    column unscaled), column K + 1 updated at once, and the candidates of step K + 1
    const bool zero = sh.zero;
    const int p = sh.p;
    const C *u = sh.u[par];
    if (zero && cx.rank == 0 && cx.tid == 0) atomicCAS(cx.info, 0, cx.j + K + 1);
    if (!zero && p != K && cx.valid) {
        if (cx.pr == K) {
#pragma unroll
            for (int q = 0; q < NB / 2; ++q) st.a[q] = u[2 * q + cx.half];
        } else if (cx.pr == p) {
#pragma unroll
            for (int q = 0; q < NB / 2; ++q) st.a[q] = sh.kin[2 * q + cx.half];
        }
    }
    const bool below = cx.valid && cx.pr > K;
    C l = czero<C>();
    if (cx.half == hk) l = zero ? st.a[qk] : cmul(st.a[qk], sh.rp);
    const C lo = shfl_xor_c(l, 1);
    if (cx.half != hk) l = lo;
    if (below && cx.half == hk) st.a[qk] = l;
    st.lp = l;
    st.key = 0ull;
    if constexpr (K + 1 < NB) {
        constexpr int hk1 = (K + 1) & 1, qk1 = (K + 1) >> 1;
        if (below && cx.half == hk1) {
            cfms(st.a[qk1], l, u[K + 1]);
            st.key = gepp_key((double)cabs1(st.a[qk1]));
        }
        gepp_reg_step<C, K + 1>(st, sh, cx);
    }
}

template <typename C>
__global__ void __launch_bounds__(GEPP_THREADS, 1)
k_panel_gepp_reg(int n, C *__restrict__ A, int64_t lda, int j, int nbj, int rpc, int *__restrict__ ipiv,
                 int *__restrict__ info, int *__restrict__ swapped, int *__restrict__ moves, PanelPack pk) {
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ GeppRegShared<C> sh;
    GeppRegCtx cx;
    cx.tid = threadIdx.x;
    cx.lane = cx.tid & 31;
    cx.warp = cx.tid >> 5;
    cx.half = cx.tid & 1;
    cx.rank = (int)cluster.block_rank();
    cx.cs = (int)cluster.num_blocks();
    cx.rpc = rpc;
    cx.nbj = nbj;
    cx.j = j;
    cx.info = info;
    const int m = n - j;
    const int r0 = cx.rank * rpc, r = cx.tid >> 1;
    cx.pr = r0 + r;
    cx.r0 = r0;
    cx.valid = r < rpc && cx.pr < m;

    GeppRegThread<C> st;
#pragma unroll
    for (int q = 0; q < NB / 2; ++q) {
        const int c = 2 * q + cx.half;
        st.a[q] = (cx.valid && c < nbj) ? A[(int64_t)(j + c) * lda + j + cx.pr] : czero<C>();
    }
    st.lp = czero<C>();
    st.key = (cx.valid && cx.half == 0) ? gepp_key((double)cabs1(st.a[0])) : 0ull;
    gepp_reg_step<C, 0>(st, sh, cx);
    // every CTA has finished reading every other CTA's slots before any CTA exits
    cluster.sync();

    // the factored rows back; complex64: the trailing update's packed A operand (L21)
    if (cx.valid) {
#pragma unroll
        for (int q = 0; q < NB / 2; ++q) {
            const int c = 2 * q + cx.half;
            if (c < nbj) A[(int64_t)(j + c) * lda + j + cx.pr] = st.a[q];
        }
    }
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (pk.a_hi) {
            // L21 rows are panel rows >= nbj (= NB here); padding rows up to a_rows / 2 are zero
            const int rest = m - nbj;
            const int pad_rows = pk.a_rows / 2;
            const int mrow = cx.pr - nbj;
            if (r < rpc && mrow >= 0 && mrow < pad_rows) {
                const bool live = mrow < rest;
#pragma unroll
                for (int q = 0; q < NB / 2; ++q) {
                    const int c = 2 * q + cx.half;
                    float xr = 0.f, xi = 0.f;
                    if (live) {
                        const float2 x = *reinterpret_cast<const float2 *>(&st.a[q]);
                        xr = x.x;
                        xi = x.y;
                    }
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow, 2 * c, pk.a_rows), xr, -xi);
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow + 1, 2 * c, pk.a_rows), xi, xr);
                }
            }
            // rows past the rows of every CTA (rpc * CS may not reach pad_rows): zero
            const int covered = cx.cs * rpc - nbj;
            if (cx.rank == 0)
                for (int e = cx.tid; e < (pad_rows - covered) * NB; e += GEPP_THREADS) {
                    const int mr = covered + e / NB, cc = e % NB;
                    if (mr < 0) continue;
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mr, 2 * cc, pk.a_rows), 0.f, 0.f);
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mr + 1, 2 * cc, pk.a_rows), 0.f, 0.f);
                }
        }
    }

    // CTA 0: ipiv, the swapped flag and the row moves of the panel's interchanges
    if (cx.rank != 0) return;
    if (cx.tid < nbj) ipiv[j + cx.tid] = j + sh.ipiv[cx.tid] + 1;
    if (cx.warp == 0) {
        const int cnt = panel_moves(sh.ipiv, nbj, j, moves, sh.first, sh.slot, sh.content, sh.extra);
        if (cx.lane == 0) *swapped = cnt > 0;
    }
}

// U12 = inv(L11) A12 of the trailing columns after the panel's row moves: one CTA per
// blockDim.x / 4 columns (UMOVES_THREADS: 32 columns), 4 threads per column, so that the
// 64-step substitution chains of a panel spread over about twice as many SMs as there are
// 64-column blocks.  Each column gathers every move's source before writing any
// destination.  complex64: also writes the trailing update's packed B operand.  Dynamic
// smem: NB * NBP + NB elements (the diagonal block and its reciprocals).
#define UMOVES_THREADS 128
template <typename C>
__global__ void __launch_bounds__(UMOVES_THREADS)
k_panel_u_moves(int n, C *__restrict__ A, int64_t lda, int j, int nbj, const int *__restrict__ moves, PanelPack pk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *T = reinterpret_cast<C *>(smem_raw);
    C *rd = T + NB * NBP;
    __shared__ int s_dst[GEPP_MAX_MOVES], s_src[GEPP_MAX_MOVES];
    __shared__ int s_cnt;
    const int t = threadIdx.x, s = t & 3, lane_vec = t >> 2;
    const int cols_per_cta = (int)blockDim.x >> 2;
    if (t == 0) s_cnt = min(moves[0], GEPP_MAX_MOVES);
    __syncthreads();
    const int cnt = s_cnt;
    for (int i = t; i < cnt; i += blockDim.x) {
        s_dst[i] = moves[1 + i];
        s_src[i] = moves[1 + GEPP_MAX_MOVES + i];
    }
    __syncthreads();
    const int col = j + nbj + cols_per_cta * blockIdx.x + lane_vec;
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
    subst_col_lower1_loop(v, T, s);
    if (ok) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = 4 * i + s;
            if (r < nbj) A[(int64_t)col * lda + j + r] = v[i];
        }
    }
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (pk.b_hi) {
            const int nb_row = cols_per_cta * blockIdx.x + lane_vec;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int r = 4 * i + s;
                pack_pair(pk.b_hi, pk.b_lo, tc_tile_offset(nb_row, 2 * r, pk.b_rows), ok ? (float)v[i].x : 0.f,
                          ok ? (float)v[i].y : 0.f);
            }
        }
    }
}
