// Tournament-pivoting panel factorization (TSLU, the panel step of communication-avoiding
// LU: Grigori, Demmel and Xiang, SIAM J. Matrix Anal. Appl. 32 (2011) 1317-1350).
//
// Partial pivoting picks each column's pivot from every remaining row of the panel, so a
// panel of 64 columns spread over many SMs costs 64 grid-wide agreements.  The tournament
// picks the panel's 64 pivot rows in a reduction tree instead:
//   * level 0: every CTA takes 128 consecutive panel rows (two threads per row, the row in
//     registers) and runs partial pivoting on them alone -- one __syncthreads per column --
//     keeping only WHICH rows it chose, in order (at most 64);
//   * merges: the chosen rows of two sibling CTAs (at most 128, their original values read
//     again from the panel) go through the same selection; the CTA that finishes a pair
//     last does the merge ("last arrival merges", counted with a global atomic), so no CTA
//     waits for another and no co-residency is needed;
//   * the root's selection is the panel's pivot order, and its in-place elimination is the
//     LU of those 64 rows (L11 and U11, the rows in pivot order, no further pivoting).
// k_tslu_finish then forms L21 = A21 inv(U11) for every other row (one substitution per
// row), moves the rows to their final places and writes the top block.  The interchanges
// are stored as LAPACK-style ipiv (a swap sequence) and as the row-move list of pivot.cuh,
// so the trailing columns, the left columns and getrs apply them exactly as they apply
// partial pivoting's.
//
// Stability: the tournament's growth factor is bounded like partial pivoting's in
// practice; on the linear-Galerkin airfoil systems of 1024 and 2048 unknowns the FP64
// backward error is 7e-14 to 1.4e-13 (partial pivoting: 1.7e-14 to 5e-14) and the
// complex64 one equal to partial pivoting's.  The pivots differ from LAPACK's.
//
// Cost (B200, ncu): a selection level takes ~2,500 cycles per column on one SM (128 rows,
// 8 warps, latency-bound at 29 % issue), so the 5 levels of a 2048-row panel take longer
// than partial pivoting's single pass over a 16-CTA cluster; the tree only pays once a
// level's column step costs well under a fifth of a cluster-wide one.  GRIM_PIVOT_TOURNAMENT
// selects it; the linear-Galerkin systems default to partial pivoting.
#pragma once
#include "pivot.cuh"

#define TSLU_ROWS 128
#define TSLU_THREADS 256
#define TSLU_WARPS (TSLU_THREADS / 32)

template <typename C>
struct TsluShared {
    C pub[2][TSLU_WARPS][2 * NB];        // [parity][warp]: the warp's best row by absolute column (upper half zero)
    C prp[2][TSLU_WARPS];                // [parity][warp]: reciprocal of its element in the step's column
    unsigned long long key[2][TSLU_WARPS];
    int slot[2][TSLU_WARPS];             // row slot of the warp's best
    int list[2 * NB];                    // slot -> panel row of the current selection
    int sel[NB];                         // chosen slots, in pivot order
    int rank_of[2 * NB];                 // slot -> its pivot step (-1: not chosen)
    int nsel, zero_first, go;
    // root: the interchange sequence and the row moves (pivot.cuh panel_moves scratch)
    int ipiv[NB], first[NB], pslot[NB], content[2 * NB], extra[NB];
    int trow[2 * NB], tpos[2 * NB];
};

// The selection runs as a loop over column pairs whose body stays in the instruction cache
// (a fully unrolled 64-column elimination is ~150 KB of straight-line code, fetched from L2
// at about a byte per cycle).  Registers are indexed by compile-time constants all the
// same: thread half h holds its row's columns h, h + 2, ... and the array is shifted down
// one register after each pair, so at pair t register q holds column 2 (q + t) + h and the
// step's column is always register 0.  The loop runs in four phases of eight pairs, phase p
// keeping LIVE = 32 - 8 p registers (columns past the panel are zero and need no work).
//
// One column step (column K = 2 t + H, owner half H): the best alive row by |re| + |im|
// (first slot on ties), published with its reciprocal pivot before the barrier; after it,
// the rank-1 update of the rows still alive.  At the root, the pivot row's columns K..nbj-1
// are row K of U11 (written to top).  Returns false once no row is left (the same in every
// thread) or past the panel.
template <typename C, int H, int LIVE>
__device__ __forceinline__ bool tslu_col(C (&a)[NB / 2], bool &alive, TsluShared<C> &sh, int t, int nbj,
                                         C *__restrict__ top) {
    const int K = 2 * t + H;
    if (K >= nbj) return false;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, half = tid & 1, slot = tid >> 1;
    unsigned long long key = 0ull;
    if (half == H && alive) {
        const double v = (double)cabs1(a[0]);
        key = v == v ? (unsigned long long)__double_as_longlong(v) + 1ull : 1ull;
    }
    unsigned long long wmax;
    const int wl = gepp_warp_argmax(key, wmax);
    if (wl >= 0 && (lane == wl || lane == (wl ^ 1))) {
        C *row = sh.pub[H][warp];
#pragma unroll
        for (int q = 0; q < LIVE; ++q) row[2 * (q + t) + half] = a[q];
        if (lane == wl) {
            const C v = a[0];
            sh.prp[H][warp] = (v.x == 0 && v.y == 0) ? czero<C>() : crecip(v);
        }
    }
    if (lane == 0) {
        sh.key[H][warp] = wl >= 0 ? wmax : 0ull;
        sh.slot[H][warp] = wl >= 0 ? (warp * 32 + wl) >> 1 : 0;
    }
    __syncthreads();
    unsigned long long g = sh.key[H][0];
    int w = 0;
#pragma unroll
    for (int u = 1; u < TSLU_WARPS; ++u)
        if (sh.key[H][u] > g) {
            g = sh.key[H][u];
            w = u;
        }
    if (g == 0ull) return false;
    const int ps = sh.slot[H][w];
    const C *u = sh.pub[H][w];
    if (tid == 0) {
        sh.sel[K] = ps;
        sh.rank_of[ps] = K;
        sh.nsel = K + 1;
        if (g == 1ull && sh.zero_first == NB) sh.zero_first = K;
    }
    if (top && tid >= K && tid < nbj) top[tid * NB + K] = u[tid];
    if (slot == ps) alive = false;
    const C rp = sh.prp[H][w];
    C l = czero<C>();
    if (half == H) l = cmul(a[0], rp);
    const C lo = shfl_xor_c(l, 1);
    if (half != H) l = lo;
    if (alive) {
        // register 0 of the other half is column K + 1 when H == 0; every other register 0
        // is column K or earlier
        if (H == 0 && half == 1) cfms(a[0], l, u[2 * t + 1]);
#pragma unroll
        for (int q = 1; q < LIVE; ++q) cfms(a[q], l, u[2 * (q + t) + half]);
    }
    return true;
}

template <typename C, int LIVE>
__device__ __forceinline__ bool tslu_phase(C (&a)[NB / 2], bool &alive, TsluShared<C> &sh, int t0, int nbj,
                                           C *__restrict__ top) {
#pragma unroll 1
    for (int t = t0; t < t0 + 8; ++t) {
        if (!tslu_col<C, 0, LIVE>(a, alive, sh, t, nbj, top)) return false;
        if (!tslu_col<C, 1, LIVE>(a, alive, sh, t, nbj, top)) return false;
#pragma unroll
        for (int q = 0; q + 1 < LIVE; ++q) a[q] = a[q + 1];
        a[LIVE - 1] = czero<C>();
    }
    return true;
}

// Selection over the nrows panel rows in sh.list: sh.sel[0..nsel) (slots in pivot order);
// with top (the root) also U11.
template <typename C>
__device__ __forceinline__ void tslu_select(const C *__restrict__ A, int64_t lda, int j, int nbj, int nrows,
                                            TsluShared<C> &sh, C *__restrict__ top) {
    const int tid = threadIdx.x, slot = tid >> 1, half = tid & 1;
    bool alive = slot < nrows;
    const int row = alive ? sh.list[slot] : 0;
    C a[NB / 2];
#pragma unroll
    for (int q = 0; q < NB / 2; ++q) {
        const int c = 2 * q + half;
        a[q] = (alive && c < nbj) ? A[(int64_t)(j + c) * lda + j + row] : czero<C>();
    }
    if (tid < 2 * NB) sh.rank_of[tid] = -1;
    if (tid == 0) {
        sh.nsel = 0;
        sh.zero_first = NB;
    }
    __syncthreads();
    if (tslu_phase<C, 32>(a, alive, sh, 0, nbj, top) && tslu_phase<C, 24>(a, alive, sh, 8, nbj, top) &&
        tslu_phase<C, 16>(a, alive, sh, 16, nbj, top))
        tslu_phase<C, 8>(a, alive, sh, 24, nbj, top);
    __syncthreads();
}

// The tournament tree of one panel (rows j..n-1, columns j..j+nbj-1 of A, left unchanged).
// Grid: ceil((n - j) / TSLU_ROWS) CTAs of TSLU_THREADS.  Node storage (reused by every
// panel): cand[node * NB + s] the node's chosen panel rows, ccount[node] their number;
// arrive[] (zero at launch, one region per panel) counts the children of each merge node
// that have finished.  Nodes of level l occupy [off_l, off_l + g_l), g_0 = grid size,
// g_{l+1} = ceil(g_l / 2); the children of node i of level l + 1 are nodes 2i and 2i + 1 of
// level l.  The root writes: top (NB x NB, column-major: U11 in its upper triangle, row s
// the pivot row of step s as eliminated), winners[s] (panel row of pivot s), ipiv (1-based, absolute), the first
// zero pivot into *info (if none earlier), *swapped and the row moves (pivot.cuh format).
template <typename C>
__global__ void __launch_bounds__(TSLU_THREADS, 1)
k_tslu_tree(int n, const C *__restrict__ A, int64_t lda, int j, int nbj, int *__restrict__ cand,
            int *__restrict__ ccount, int *__restrict__ arrive, C *__restrict__ top, int *__restrict__ winners,
            int *__restrict__ ipiv, int *__restrict__ info, int *__restrict__ swapped, int *__restrict__ moves) {
    __shared__ TsluShared<C> sh;
    const int tid = threadIdx.x;
    const int m = n - j;
    int gl = (int)gridDim.x, off = 0, node = (int)blockIdx.x;
    const int r0 = node * TSLU_ROWS;
    int nrows = min(TSLU_ROWS, m - r0);
    for (int s = tid; s < nrows; s += TSLU_THREADS) sh.list[s] = r0 + s;
    __syncthreads();
    while (true) {
        tslu_select<C>(A, lda, j, nbj, nrows, sh, gl == 1 ? top : nullptr);
        const int nsel = sh.nsel;
        if (gl == 1) break;  // this CTA holds the root
        int *mine = cand + (size_t)(off + node) * NB;
        for (int s = tid; s < nsel; s += TSLU_THREADS) mine[s] = sh.list[sh.sel[s]];
        if (tid == 0) ccount[off + node] = nsel;
        __threadfence();
        __syncthreads();
        const int parent = node >> 1;
        const int nchild = min(2, gl - 2 * parent);
        if (tid == 0) {
            const int old = atomicAdd(&arrive[off + gl + parent], 1);
            sh.go = old == nchild - 1;
            __threadfence();
        }
        __syncthreads();
        if (!sh.go) return;  // the sibling merges
        int cnt = 0;
        for (int ch = 2 * parent; ch < 2 * parent + nchild; ++ch) {
            const int cn = __ldcg(&ccount[off + ch]);
            for (int s = tid; s < cn; s += TSLU_THREADS) sh.list[cnt + s] = __ldcg(&cand[(size_t)(off + ch) * NB + s]);
            cnt += cn;
        }
        __syncthreads();
        nrows = cnt;
        node = parent;
        off += gl;
        gl = (gl + 1) >> 1;
    }

    // root: the pivot rows, the interchanges and the row moves (U11 is in top)
    const int nsel = sh.nsel;  // == nbj (every panel has at least nbj rows)
    if (tid < nsel) winners[tid] = sh.list[sh.sel[tid]];
    if (tid == 0 && sh.zero_first < nbj) atomicCAS(info, 0, j + sh.zero_first + 1);
    __syncthreads();
    if (tid >= 32) return;
    // the swap sequence that brings pivot row s to place s, simulated on the touched places:
    // entries e < nbj are places 0..nbj-1, later entries the places of pivot rows >= nbj
    const int lane = tid;
    for (int e = lane; e < nbj; e += 32) {
        sh.tpos[e] = e;
        sh.trow[e] = e;
    }
    int nt = nbj;
    for (int s0 = 0; s0 < nbj; s0 += 32) {
        const int s = s0 + lane;
        const int w = s < nbj ? sh.list[sh.sel[s]] : 0;
        const bool ext = s < nbj && w >= nbj;
        const unsigned bal = __ballot_sync(0xffffffffu, ext);
        if (ext) {
            const int e = nt + __popc(bal & ((1u << lane) - 1u));
            sh.tpos[e] = w;
            sh.trow[e] = w;
        }
        nt += __popc(bal);
    }
    __syncwarp();
    for (int s = 0; s < nbj; ++s) {
        const int w = sh.list[sh.sel[s]];
        int found = -1;
        for (int e0 = 0; e0 < nt; e0 += 32) {
            const int e = e0 + lane;
            const unsigned b = __ballot_sync(0xffffffffu, e < nt && sh.trow[e] == w);
            if (b) {
                found = e0 + __ffs(b) - 1;
                break;
            }
        }
        __syncwarp();
        if (found < 0) found = s;  // cannot happen: every pivot row is in the table
        if (lane == 0) {
            const int p = sh.tpos[found];
            sh.ipiv[s] = p;
            const int t = sh.trow[s];
            sh.trow[s] = sh.trow[found];
            sh.trow[found] = t;
        }
        __syncwarp();
    }
    for (int s = lane; s < nbj; s += 32) ipiv[j + s] = j + sh.ipiv[s] + 1;
    const int cntm = panel_moves(sh.ipiv, nbj, j, moves, sh.first, sh.pslot, sh.content, sh.extra);
    if (lane == 0) *swapped = cntm > 0;
}

// After k_tslu_tree: every panel row gets x = a inv(U11) (its original panel row a, one row
// substitution x U11 = a per row, four lanes per row).  A row that is not a pivot row is
// L21's row x, written to its final place (the row moves' destination, else its own
// place).  Pivot row s becomes row s of the top block: x in columns < s (L11's row, which
// x U11 = a gives for a row whose elimination used the pivots before it) and U11's row s
// (from top) in columns >= s.  Only CTA 0 writes places 0..nbj-1 and the pivot rows' old
// places, and it reads the rows it overwrites (its own rows 0..nbj-1 and the pivot rows)
// before writing any of them; the other CTAs write only their own non-pivot rows in place.
// Grid: as k_tslu_tree.  complex64 with pk.a_hi: also the trailing update's packed A operand
// (L21 by final place, rows past the panel zero up to pk.a_rows / 2).  Dynamic smem:
// (NB * NBP + NB) elements.
template <typename C>
__global__ void __launch_bounds__(256)
k_tslu_finish(int n, C *__restrict__ A, int64_t lda, int j, int nbj, const C *__restrict__ top,
              const int *__restrict__ winners, const int *__restrict__ moves, PanelPack pk) {
    extern __shared__ __align__(16) unsigned char tslu_smem[];
    C *T = reinterpret_cast<C *>(tslu_smem);  // U11, padded (NB * NBP), then the reciprocals
    C *rd = T + NB * NBP;                      // of its diagonal (NB)
    __shared__ int s_dst[GEPP_MAX_MOVES], s_src[GEPP_MAX_MOVES];
    __shared__ int is_win[TSLU_ROWS], dst_of[TSLU_ROWS];
    const int tid = threadIdx.x;
    const int m = n - j;
    const int r0 = blockIdx.x * TSLU_ROWS;
    const int cnt = min(moves[0], GEPP_MAX_MOVES);
    for (int i = tid; i < cnt; i += 256) {
        s_dst[i] = moves[1 + i] - j;
        s_src[i] = moves[1 + GEPP_MAX_MOVES + i] - j;
    }
    for (int i = tid; i < TSLU_ROWS; i += 256) {
        is_win[i] = 0;
        dst_of[i] = r0 + i;
    }
    for (int e = tid; e < NB * NB; e += 256) {
        const int r = e & (NB - 1), c = e >> 6;
        T[c * NBP + r] = (r <= c && r < nbj && c < nbj) ? top[c * NB + r] : czero<C>();
    }
    __syncthreads();
    if (tid < nbj) {
        const C d = top[tid * NB + tid];
        rd[tid] = (d.x == 0 && d.y == 0) ? czero<C>() : crecip(d);
        const int w = winners[tid] - r0;
        if (w >= 0 && w < TSLU_ROWS) is_win[w] = 1;
    }
    for (int i = tid; i < cnt; i += 256) {
        const int s = s_src[i] - r0;
        if (s >= 0 && s < TSLU_ROWS) dst_of[s] = s_dst[i];
    }
    if (tid >= nbj && tid < NB) rd[tid] = one_c<C>();
    __syncthreads();
    const int sub = tid & 3, rr = tid >> 2;
    const int rest = m - nbj;
    // CTA 0: the pivot rows' L11 parts first (kept in registers until the end)
    C xw[16];
    const bool win_row = blockIdx.x == 0 && rr < nbj;
    if (blockIdx.x == 0) {
        const int w = win_row ? winners[rr] : 0;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int c = 4 * i + sub;
            xw[i] = (win_row && c < rr) ? A[(int64_t)(j + c) * lda + j + w] : czero<C>();
        }
        subst_row_upper_loop(xw, T, rd, nbj, sub);
        __syncthreads();  // every pivot row read before any place is written
    }
    for (int pass = 0; pass < TSLU_ROWS / 64; ++pass) {
        const int li = pass * 64 + rr;
        const int r = r0 + li;
        const bool valid = r < m && !is_win[li];
        C v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int c = 4 * i + sub;
            v[i] = (valid && c < nbj) ? A[(int64_t)(j + c) * lda + j + r] : czero<C>();
        }
        subst_row_upper_loop(v, T, rd, nbj, sub);
        // a row that is not a pivot row goes to its own place or (rows 0..nbj-1 of CTA 0) to a
        // pivot row's old place, which no thread reads any more
        const int d = valid ? dst_of[li] : 0;
        if (valid) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int c = 4 * i + sub;
                if (c < nbj) A[(int64_t)(j + c) * lda + j + d] = v[i];
            }
        }
        if constexpr (sizeof(C) == sizeof(float2)) {
            if (pk.a_hi && valid && d >= nbj) {
                const int mrow = d - nbj;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int c = 4 * i + sub;
                    const float2 x = *reinterpret_cast<const float2 *>(&v[i]);
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow, 2 * c, pk.a_rows), x.x, -x.y);
                    pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mrow + 1, 2 * c, pk.a_rows), x.y, x.x);
                }
            }
        }
    }
    if (blockIdx.x != 0) return;
    __syncthreads();  // CTA 0's rows 0..nbj-1 read before the top block is written
    if (win_row) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int c = 4 * i + sub;
            if (c < nbj) A[(int64_t)(j + c) * lda + j + rr] = c < rr ? xw[i] : top[c * NB + rr];
        }
    }
    if constexpr (sizeof(C) == sizeof(float2)) {
        if (pk.a_hi) {
            const int pad_rows = pk.a_rows / 2;
            for (int e = tid; e < (pad_rows - rest) * NB; e += 256) {
                const int mr = rest + e / NB, cc = e % NB;
                pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mr, 2 * cc, pk.a_rows), 0.f, 0.f);
                pack_pair(pk.a_hi, pk.a_lo, tc_tile_offset(2 * mr + 1, 2 * cc, pk.a_rows), 0.f, 0.f);
            }
        }
    }
}
