// Partial-pivoting panel factorization on a thread-block cluster, loop-resident form.
//
// The same factorization as k_panel_gepp_reg (LAPACK getf2's pivots: |re| + |im|, first
// position on ties; one cluster barrier per column), restructured so that its column loop
// runs from the instruction cache.  The unrolled kernel spends most of a column step
// waiting for instructions (~4 KB of straight-line code per column, fetched from L2); here
// a pair of columns is one loop iteration:
//   * rows never move during the panel: each row stays in the registers of its two threads
//     (thread half h holding columns h, h + 2, ...) and carries its current position, so an
//     interchange is two position updates; the rows are written to their final places at
//     the end;
//   * after each pair the row registers shift down one, so register q holds column
//     2 (q + t) + h at pair t and every register index is a compile-time constant;
//     finished columns (multipliers, pivots, U entries) retire to shared memory;
//   * the loop runs in four phases of eight pairs keeping 32, 24, 16 and 8 registers.
// Column step K (owner half H = K & 1, its value in register 0):
//   1. the CTA's best alive row (largest key, then lowest position), published with its
//      pending multiplier and pushed as a candidate (key, position, element) into every
//      CTA of the cluster;
//   2. the cluster barrier, with step K - 1's rank-1 update of columns > K applied while the
//      other CTAs arrive;
//   3. warp 0 picks the winner among the candidates, reads its row through distributed
//      shared memory and applies that row's pending update;
//   4. every row: position update, multiplier, column K retired, column K + 1 updated at
//      once (the next step's candidates), the rest deferred to the next step.
// Double-buffered slots are rewritten two steps later, after every CTA has passed the
// cluster barrier that follows their last reads.
#pragma once
#include "pivot.cuh"

#define GEPPL_THREADS 256
#define GEPPL_ROWS (GEPPL_THREADS / 2)
#define GEPPL_WARPS (GEPPL_THREADS / 32)

template <typename C>
struct GeppLCand {
    C piv;                   // the candidate's element in the step's column
    C lp;                    // its pending multiplier (the previous step's)
    unsigned long long key;  // 0: no candidate
    int pos;                 // its current position in the panel
    int pad;
};

template <typename C>
struct GeppLShared {
    C pub[2][2 * NB];  // [parity]: the CTA's best row by absolute column (pending values)
    C pub_lp[2];       // [parity]: its pending multiplier
    C u[2][2 * NB];    // [parity]: the step's pivot row, columns > K (upper half zero)
    GeppLCand<C> cand[2][16];
    unsigned long long wkey[2][GEPPL_WARPS];
    int wpos[2][GEPPL_WARPS], wslot[2][GEPPL_WARPS];
    C rp;
    int wp, zero;
    int ipiv[NB], first[NB], pslot[NB], content[2 * NB], extra[NB];
};

struct GeppLCtx {
    int tid, lane, warp, half, slot, rank, cs, nbj, j;
    int *info;
};

template <typename C>
struct GeppLRow {
    C a[NB / 2];
    C lp;  // multiplier of the previous step, still to be applied to columns > K
    int pos;
    bool alive, valid;
};

// Warp maximum of the keys, then the lowest position among the lanes that hold it: returns
// that lane (-1 when every key is 0) and the maximum key (every lane).
__device__ __forceinline__ int geppl_warp_best(unsigned long long key, int pos, unsigned long long &kmax) {
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    kmax = ((unsigned long long)mhi << 32) | mlo;
    const bool top = kmax != 0ull && key == kmax;
    const unsigned pmin = __reduce_min_sync(0xffffffffu, top ? (unsigned)pos : 0xffffffffu);
    const unsigned bal = __ballot_sync(0xffffffffu, top && (unsigned)pos == pmin);
    return bal ? __ffs(bal) - 1 : -1;
}

// PUSH: every CTA pushes its candidate row (the live columns) into every CTA before the
// cluster barrier, so the winner's row is read from local shared memory afterwards (crow:
// [parity][rank][2 NB] elements of dynamic shared memory) instead of through a distributed
// shared-memory load after it.
template <typename C, int H, int LIVE, bool PUSH>
__device__ __forceinline__ void geppl_col(GeppLRow<C> &st, GeppLShared<C> &sh, C *__restrict__ retired,
                                          C *__restrict__ crow, const GeppLCtx &cx, int t) {
    const int K = 2 * t + H;
    if (K >= cx.nbj) return;
    cg::cluster_group cluster = cg::this_cluster();
    const C *uprev = sh.u[H ^ 1];

    // 1. the warp's and then the CTA's best alive row for column K
    unsigned long long key = 0ull;
    int pos = 0x7fffffff;
    if (cx.half == H && st.alive) {
        key = gepp_key((double)cabs1(st.a[0]));
        pos = st.pos;
    }
    unsigned long long wmax;
    const int wl = geppl_warp_best(key, pos, wmax);
    const int wpos = __shfl_sync(0xffffffffu, pos, wl >= 0 ? wl : 0);
    if (cx.lane == 0) {
        sh.wkey[H][cx.warp] = wl >= 0 ? wmax : 0ull;
        sh.wpos[H][cx.warp] = wl >= 0 ? wpos : 0x7fffffff;
        sh.wslot[H][cx.warp] = wl >= 0 ? (cx.warp * 32 + wl) >> 1 : 0;
    }
    __syncthreads();
    unsigned long long ck = sh.wkey[H][0];
    int cp = sh.wpos[H][0], cw = 0;
#pragma unroll
    for (int w = 1; w < GEPPL_WARPS; ++w) {
        const unsigned long long k2 = sh.wkey[H][w];
        const int p2 = sh.wpos[H][w];
        if (k2 > ck || (k2 == ck && p2 < cp)) {
            ck = k2;
            cp = p2;
            cw = w;
        }
    }
    const int cslot = sh.wslot[H][cw];
    // its row published (pending values and multiplier), its candidate pushed into every CTA
    // by its warp (warp 0 pushes "no candidate" when the CTA has none)
    if (ck != 0ull && cx.slot == cslot) {
#pragma unroll
        for (int q = 0; q < LIVE; ++q) sh.pub[H][2 * (q + t) + cx.half] = st.a[q];
        if (cx.half == 0) sh.pub_lp[H] = st.lp;
    }
    const int ow = ck != 0ull ? (2 * cslot) >> 5 : 0;
    if (cx.warp == ow) {
        const C piv = shfl_c(st.a[0], (2 * cslot + H) & 31);
        const C plp = shfl_c(st.lp, (2 * cslot) & 31);
        if (PUSH && ck != 0ull) {
            // the row's live columns [2 t, 2 t + 2 LIVE) into every CTA's slot for this rank
            __syncwarp();
            for (int e = cx.lane; e < cx.cs * 2 * LIVE; e += 32) {
                const int d = e / (2 * LIVE), c = 2 * t + e % (2 * LIVE);
                *cluster.map_shared_rank(&crow[(H * 16 + cx.rank) * 2 * NB + c], d) = sh.pub[H][c];
            }
        }
        if (cx.lane < cx.cs) {
            GeppLCand<C> c;
            c.piv = piv;
            c.lp = plp;
            c.key = ck;
            c.pos = cp;
            c.pad = 0;
            *cluster.map_shared_rank(&sh.cand[H][cx.rank], cx.lane) = c;
        }
    }
    __syncwarp();
    gepp_arrive(cx.warp == ow);

    // 2. step K - 1's update of columns > K while the other CTAs arrive
    if (st.alive && K > 0) {
        if (H == 0 && cx.half == 1) cfms(st.a[0], st.lp, uprev[2 * t + 1]);
#pragma unroll
        for (int q = 1; q < LIVE; ++q) cfms(st.a[q], st.lp, uprev[2 * (q + t) + cx.half]);
    }
    __syncwarp();
    gepp_wait();

    // 3. warp 0: the winner (largest key, then lowest position) and its row, columns > K
    if (cx.warp == 0) {
        unsigned long long k1 = 0ull;
        int p1 = 0x7fffffff;
        if (cx.lane < cx.cs) {
            k1 = sh.cand[H][cx.lane].key;
            p1 = sh.cand[H][cx.lane].pos;
        }
        unsigned long long gmax;
        const int wr = geppl_warp_best(k1, p1, gmax);
        const bool zero = gmax <= 1ull;  // every candidate 0 (or none): no elimination
        const int c0 = cx.lane, c1 = cx.lane + 32;
        C x0 = czero<C>(), x1 = czero<C>();
        if (wr >= 0) {
            const C *wrow = PUSH ? crow + (H * 16 + wr) * 2 * NB : cluster.map_shared_rank(&sh.pub[H][0], wr);
            const C wlp = PUSH ? sh.cand[H][wr].lp : *cluster.map_shared_rank(&sh.pub_lp[H], wr);
            if (c0 > K) {
                x0 = wrow[c0];
                if (K > 0) cfms(x0, wlp, uprev[c0]);
            }
            if (c1 > K) {
                x1 = wrow[c1];
                if (K > 0) cfms(x1, wlp, uprev[c1]);
            }
        }
        sh.u[H][c0] = x0;
        sh.u[H][c1] = x1;
        if (cx.lane == 0) {
            const int wp = wr >= 0 ? sh.cand[H][wr].pos : K;
            sh.wp = wp;
            sh.zero = zero;
            sh.rp = zero ? czero<C>() : crecip(sh.cand[H][wr].piv);
            if (cx.rank == 0) {
                sh.ipiv[K] = wp;
                if (zero) atomicCAS(cx.info, 0, cx.j + K + 1);
            }
        }
    }
    __syncthreads();

    // 4. positions, multipliers, column K retired, column K + 1 updated at once
    const int wp = sh.wp;
    const bool zero = sh.zero;
    const C rp = sh.rp;
    const C *u = sh.u[H];
    if (st.alive) {
        if (st.pos == wp) {
            st.alive = false;  // the pivot row: position K, its values final
            st.pos = K;
        } else if (st.pos == K) {
            st.pos = wp;
        }
    }
    C l = czero<C>();
    if (cx.half == H) l = zero ? st.a[0] : cmul(st.a[0], rp);
    const C lo = shfl_xor_c(l, 1);
    if (cx.half != H) l = lo;
    if (cx.half == H) retired[K * GEPPL_ROWS + cx.slot] = st.alive ? l : st.a[0];
    if (st.alive) {
        if (H == 0 && cx.half == 1) cfms(st.a[0], l, u[K + 1]);
        if (H == 1 && cx.half == 0) cfms(st.a[1], l, u[K + 1]);
        st.lp = l;
    } else {
        st.lp = czero<C>();
    }
}

template <typename C, int LIVE, bool PUSH>
__device__ __forceinline__ void geppl_phase(GeppLRow<C> &st, GeppLShared<C> &sh, C *__restrict__ retired,
                                            C *__restrict__ crow, const GeppLCtx &cx, int t0) {
#pragma unroll 1
    for (int t = t0; t < t0 + 8; ++t) {
        if (2 * t >= cx.nbj) return;  // the same in every thread
        geppl_col<C, 0, LIVE, PUSH>(st, sh, retired, crow, cx, t);
        geppl_col<C, 1, LIVE, PUSH>(st, sh, retired, crow, cx, t);
#pragma unroll
        for (int q = 0; q + 1 < LIVE; ++q) st.a[q] = st.a[q + 1];
        st.a[LIVE - 1] = czero<C>();
    }
}

// The panel (j, nbj) of A, rows j..n-1, on a cluster of gridDim.x CTAs, CTA c holding panel
// rows [c rpc, (c + 1) rpc) (rpc <= GEPPL_ROWS).  Dynamic smem: NB * GEPPL_ROWS elements
// (the retired columns, column-major by row slot), then with PUSH 2 x 16 x 2 NB elements (the
// pushed candidate rows).  Outputs as k_panel_gepp_reg: the factored
// panel in place, ipiv (1-based, absolute), the first zero pivot in *info, *swapped, the
// row moves, and (complex64, pk.a_hi) the trailing update's packed L21 operand.
template <typename C, bool PUSH>
__global__ void __launch_bounds__(GEPPL_THREADS, 1)
k_panel_gepp_loop(int n, C *__restrict__ A, int64_t lda, int j, int nbj, int rpc, int *__restrict__ ipiv,
                  int *__restrict__ info, int *__restrict__ swapped, int *__restrict__ moves, PanelPack pk) {
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ GeppLShared<C> sh;
    extern __shared__ __align__(16) unsigned char geppl_smem[];
    C *retired = reinterpret_cast<C *>(geppl_smem);
    C *crow = retired + NB * GEPPL_ROWS;
    GeppLCtx cx;
    cx.tid = threadIdx.x;
    cx.lane = cx.tid & 31;
    cx.warp = cx.tid >> 5;
    cx.half = cx.tid & 1;
    cx.slot = cx.tid >> 1;
    cx.rank = (int)cluster.block_rank();
    cx.cs = (int)cluster.num_blocks();
    cx.nbj = nbj;
    cx.j = j;
    cx.info = info;
    const int m = n - j;
    GeppLRow<C> st;
    st.pos = cx.rank * rpc + cx.slot;
    st.valid = cx.slot < rpc && st.pos < m;
    st.alive = st.valid;
    st.lp = czero<C>();
#pragma unroll
    for (int q = 0; q < NB / 2; ++q) {
        const int c = 2 * q + cx.half;
        st.a[q] = (st.valid && c < nbj) ? A[(int64_t)(j + c) * lda + j + st.pos] : czero<C>();
    }
    for (int e = cx.tid; e < 2 * 2 * NB; e += GEPPL_THREADS) (&sh.u[0][0])[e] = czero<C>();
    for (int e = cx.tid; e < NB * GEPPL_ROWS; e += GEPPL_THREADS) retired[e] = czero<C>();
    // every CTA's slots initialised before any CTA pushes into them
    cluster.sync();
    geppl_phase<C, 32, PUSH>(st, sh, retired, crow, cx, 0);
    geppl_phase<C, 24, PUSH>(st, sh, retired, crow, cx, 8);
    geppl_phase<C, 16, PUSH>(st, sh, retired, crow, cx, 16);
    geppl_phase<C, 8, PUSH>(st, sh, retired, crow, cx, 24);
    // every CTA has finished reading every other CTA's slots before any CTA exits; the rows'
    // final places may be in other CTAs' ranges, whose rows were all read at the start
    cluster.sync();

    const int rest = m - nbj;
    if (st.valid) {
        const int d = st.pos;
        for (int c = cx.half; c < nbj; c += 2) A[(int64_t)(j + c) * lda + j + d] = retired[c * GEPPL_ROWS + cx.slot];
        if constexpr (sizeof(C) == sizeof(float2)) {
            if (pk.a_hi && d >= nbj) {
                const int mrow = d - nbj;
                for (int c = cx.half; c < NB; c += 2) {
                    float xr = 0.f, xi = 0.f;
                    if (c < nbj) {
                        const float2 x = *reinterpret_cast<const float2 *>(&retired[c * GEPPL_ROWS + cx.slot]);
                        xr = x.x;
                        xi = x.y;
                    }
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow, 2 * c, pk.a_rows), xr, -xi);
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow + 1, 2 * c, pk.a_rows), xi, xr);
                }
            }
        }
    }
    if (cx.rank != 0) return;
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (pk.a_hi) {
            // padding rows of the packed operand past the panel's rows: zero
            const int pad_rows = pk.a_rows / 2;
            for (int e = cx.tid; e < (pad_rows - rest) * NB; e += GEPPL_THREADS) {
                const int mr = rest + e / NB, cc = e % NB;
                pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mr, 2 * cc, pk.a_rows), 0.f, 0.f);
                pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mr + 1, 2 * cc, pk.a_rows), 0.f, 0.f);
            }
        }
    }
    // CTA 0: ipiv, the swapped flag and the row moves of the panel's interchanges
    if (cx.tid < nbj) ipiv[j + cx.tid] = j + sh.ipiv[cx.tid] + 1;
    if (cx.warp == 0) {
        const int cnt = panel_moves(sh.ipiv, nbj, j, moves, sh.first, sh.pslot, sh.content, sh.extra);
        if (cx.lane == 0) *swapped = cnt > 0;
    }
}
