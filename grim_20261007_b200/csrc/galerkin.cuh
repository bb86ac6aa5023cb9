// Linear-Galerkin combined-field fill of closed perfectly conducting contours: the
// reference's own 2-D discretisation (tools/GHOST/ghost_backend/twod/...), on the GPU.
//
// Elements are straight, with linear (hat) bases on their two nodes; a closed contour of
// N elements has N nodes and N unknowns.  With G = (j/4) H0^(2)(k r) the element-pair
// blocks are (r = x_obs - y_src, L the element lengths, t the parent parameters)
//   S_ab  = L_o L_s  int int phi_a(t) phi_b(s) G(r)
//   K'_ab = L_o L_s  int int phi_a phi_b  (-(j/4) k H1^(2)(k r)) (r . n_o)/|r|   (observation normal)
//   D_ab  = L_o L_s  int int phi_a phi_b  (+(j/4) k H1^(2)(k r)) (r . n_s)/|r|   (source normal)
//   W     = -k^2 (n_o . n_s) S + [[1,-1],[-1,1]] sum(S) / (L_o L_s)              (Maue form)
// and the combined rows of a PEC contour in air (twod/formulations/combined_regions.py:
// 21-62,149-204, regions.py:283-292), gamma = 1/(j k):
//   TM (Dirichlet trace)  A = S + gamma (D + M/2)
//   TE (flux)             A = K' - M/2 - gamma W
// M the consistent mass L [[1/3,1/6],[1/6,1/3]] per element.
//
// Pair routing follows twod/operators.py:2087 _assemble_multi and
// twod/assembly/separation.py:67:
//   far   : centre distance >= 3 max(L_o, L_s), no shared node: Gauss tensor rule of the
//           order the reference's calibrated table gives for the worst pair of the tile
//           (operators.py:1443-1531 _FAR_ORDER_TABLE, _graded_far_order, _graded_w_far_floor);
//           the table promises every block within 1e-12 of a converged rule, so this
//           build's own tiles (32 x 32 elements) give the reference's blocks to that level;
//   self  : closed-form small-argument series of the log-singular kernel (operators.py:418),
//           composite sub-interval rule beyond |k L| = 8 (operators.py:980);
//   touch : elements sharing a node, two triangles at the corner graded as t^4, 20-point
//           Gauss per direction (operators.py:629);
//   close : the adaptive four-way bisection to 1e-9 (operators.py:1172) when the
//           separation test asks for it, else a 16-point tensor rule (operators.py:223).
//
// Pipeline (all on the handle's stream; geometry-only steps cached by the caller):
//   k_gal_near_count / k_gal_near_list  near-pair list per element row (CSR, columns ascending)
//   k_gal_near                          S and K' of every near pair, one warp per pair (FP64)
//   k_gal_far                           far pairs of the upper tile triangle, both orientations
//                                       from one set of Hankel evaluations, routed blocks E[e][f]
//   k_gal_near_route                    routed blocks of the near pairs (+ mass on self pairs)
//   k_gal_gather                        node matrix Z[i][j] from the four element pairs of (i, j)
//   k_gal_rhs / k_gal_farfield          Galerkin plane-wave loads and the monostatic far field
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "hankel.cuh"

#define GAL_FAR_RATIO 3.0
#define GAL_EPS 1e-12
#define GAL_TOUCH_ORDER 20
#define GAL_BOX_ORDER 16
#define GAL_ADAPT_RTOL 1e-9
#define GAL_ADAPT_DEPTH 12
#define GAL_ADAPT_STACK 64
#define GAL_SERIES_LIMIT 8.0
#define GAL_SUB_KL 2.0
#define GAL_TILE 32
#define GAL_FAR_THREADS 256
#define GAL_NEAR_WARPS 4
#define GAL_LOAD_ORDER 8
#define GAL_X_ASYM 25.0
#define GAL_ASYM64_TERMS 16

#define GAL_ROUTE_SELF 0
#define GAL_ROUTE_TOUCH 1
#define GAL_ROUTE_BOX 2
#define GAL_ROUTE_ADAPT 3

// Element record, 8 doubles: start point (ax, ay), end point (bx, by), unit normal
// (nx, ny) = (-t_y, t_x) of the tangent t = (b - a)/L, length L, unused.
struct GalElem {
    double ax, ay, bx, by, nx, ny, len, pad;
};

// Hankel asymptotic coefficients a_k(0), a_k(1), k < GAL_ASYM64_TERMS (DLMF 10.17.1),
// uploaded with the other tables.
__constant__ double c_gal_a0[GAL_ASYM64_TERMS];
__constant__ double c_gal_a1[GAL_ASYM64_TERMS];

__device__ __forceinline__ GalElem gal_load(const double *elem, int e) {
    const double2 *p = (const double2 *)(elem + 8 * (size_t)e);
    const double2 u = __ldg(p), v = __ldg(p + 1), w = __ldg(p + 2), z = __ldg(p + 3);
    GalElem g;
    g.ax = u.x; g.ay = u.y; g.bx = v.x; g.by = v.y;
    g.nx = w.x; g.ny = w.y; g.len = z.x; g.pad = z.y;
    return g;
}

// Gauss-Legendre rule of order q on [0, 1] (from the [-1, 1] tables in constant memory).
__device__ __forceinline__ void gal_gauss(int q, int i, double &t, double &w) {
    const int off = q * (q - 1) / 2 + i;
    t = 0.5 * (c_gl_x[off] + 1.0);
    w = 0.5 * c_gl_w[off];
}

// ------------------------------------------------------------------ routing
__device__ __forceinline__ bool gal_shares(int2 a, int2 b) {
    return a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y;
}

// Centre distance over the longer length (the reference's far-pair ratio).
__device__ __forceinline__ double gal_ratio(const GalElem &o, const GalElem &s) {
    const double dx = 0.5 * (o.ax + o.bx) - 0.5 * (s.ax + s.bx);
    const double dy = 0.5 * (o.ay + o.by) - 0.5 * (s.ay + s.by);
    return sqrt(dx * dx + dy * dy) / fmax(fmax(o.len, s.len), GAL_EPS);
}

__device__ __forceinline__ bool gal_is_far(const GalElem &o, const GalElem &s, int2 no, int2 ns, int e, int f) {
    return e != f && !gal_shares(no, ns) && gal_ratio(o, s) >= GAL_FAR_RATIO;
}

__device__ __forceinline__ double gal_pt_seg_sq(double px, double py, double ax, double ay, double bx, double by) {
    const double ex = bx - ax, ey = by - ay;
    const double den = ex * ex + ey * ey;
    double t = den > 0.0 ? ((px - ax) * ex + (py - ay) * ey) / den : 0.0;
    t = fmin(fmax(t, 0.0), 1.0);
    const double dx = px - ax - t * ex, dy = py - ay - t * ey;
    return dx * dx + dy * dy;
}

// Distance between two closed segments, 0 when they cross.
__device__ double gal_segment_distance(const GalElem &p, const GalElem &q) {
    double sq = gal_pt_seg_sq(p.ax, p.ay, q.ax, q.ay, q.bx, q.by);
    sq = fmin(sq, gal_pt_seg_sq(p.bx, p.by, q.ax, q.ay, q.bx, q.by));
    sq = fmin(sq, gal_pt_seg_sq(q.ax, q.ay, p.ax, p.ay, p.bx, p.by));
    sq = fmin(sq, gal_pt_seg_sq(q.bx, q.by, p.ax, p.ay, p.bx, p.by));
    const double ux = p.bx - p.ax, uy = p.by - p.ay, vx = q.bx - q.ax, vy = q.by - q.ay;
    const double wx = q.ax - p.ax, wy = q.ay - p.ay;
    const double den = ux * vy - uy * vx;
    if (den != 0.0) {
        const double t = (wx * vy - wy * vx) / den, s = (wx * uy - wy * ux) / den;
        if (t >= 0.0 && t <= 1.0 && s >= 0.0 && s <= 1.0) return 0.0;
    }
    return sqrt(fmax(sq, 0.0));
}

// Smallest distance from an end of one segment to the other's interior (foot strictly inside).
__device__ double gal_projection_distance(const GalElem &p, const GalElem &q) {
    double best = INFINITY;
    const double px[4] = {p.ax, p.bx, q.ax, q.bx}, py[4] = {p.ay, p.by, q.ay, q.by};
    for (int i = 0; i < 4; ++i) {
        const GalElem &g = i < 2 ? q : p;
        const double ex = g.bx - g.ax, ey = g.by - g.ay;
        const double den = ex * ex + ey * ey;
        const double t = den > 0.0 ? ((px[i] - g.ax) * ex + (py[i] - g.ay) * ey) / den : -1.0;
        if (t > 0.0 && t < 1.0) {
            const double dx = px[i] - g.ax - t * ex, dy = py[i] - g.ay - t * ey;
            best = fmin(best, sqrt(dx * dx + dy * dy));
        }
    }
    return best;
}

// The reference's choice between the adaptive and the fixed rule for a separated near pair.
__device__ bool gal_needs_adaptive(const GalElem &o, const GalElem &s) {
    const double lo = o.len, ls = s.len, scale = fmax(lo, ls);
    const double dx = 0.5 * (o.ax + o.bx) - 0.5 * (s.ax + s.bx);
    const double dy = 0.5 * (o.ay + o.by) - 0.5 * (s.ay + s.by);
    const double dist = sqrt(dx * dx + dy * dy);
    if (dist < 0.75 * scale) return true;
    if (dist >= 0.5 * (lo + ls) + 0.5 * scale) return false;
    if (dist < 0.5 * (lo + ls) + 0.25 * scale && gal_segment_distance(o, s) < 0.25 * scale) return true;
    return gal_projection_distance(o, s) < 0.5 * scale;
}

__device__ __forceinline__ int gal_route(const GalElem &o, const GalElem &s, int2 no, int2 ns, int e, int f) {
    if (e == f) return GAL_ROUTE_SELF;
    if (gal_shares(no, ns)) return GAL_ROUTE_TOUCH;
    return gal_needs_adaptive(o, s) ? GAL_ROUTE_ADAPT : GAL_ROUTE_BOX;
}

// Near-pair count of every element row: one warp per row, 32 columns per step.
__global__ void k_gal_near_count(int ne, const double *__restrict__ elem, const int2 *__restrict__ nodes,
                                 int *__restrict__ count) {
    const int lane = threadIdx.x & 31;
    const int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (e >= ne) return;
    const GalElem o = gal_load(elem, e);
    const int2 no = nodes[e];
    int total = 0;
    for (int f0 = 0; f0 < ne; f0 += 32) {
        const int f = f0 + lane;
        bool near = false;
        if (f < ne) near = !gal_is_far(o, gal_load(elem, f), no, nodes[f], e, f);
        total += __popc(__ballot_sync(0xffffffffu, near));
    }
    if (lane == 0) count[e] = total;
}

// Exclusive prefix sum of the row counts (one CTA of 1024 threads, chunked), row_off[ne]
// the total.
__global__ void k_gal_scan(int ne, const int *__restrict__ count, int *__restrict__ row_off) {
    __shared__ int part[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ne; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < ne ? count[i] : 0;
        part[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const int add = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
            __syncthreads();
            part[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < ne) row_off[i] = carry + part[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += part[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) row_off[ne] = carry;
}

// Near-pair columns (ascending) and routes of every row.
__global__ void k_gal_near_list(int ne, const double *__restrict__ elem, const int2 *__restrict__ nodes,
                                const int *__restrict__ row_off, int *__restrict__ col, int *__restrict__ route) {
    const int lane = threadIdx.x & 31;
    const int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (e >= ne) return;
    const GalElem o = gal_load(elem, e);
    const int2 no = nodes[e];
    int pos = row_off[e];
    for (int f0 = 0; f0 < ne; f0 += 32) {
        const int f = f0 + lane;
        bool near = false;
        GalElem s;
        int2 ns = make_int2(-1, -1);
        if (f < ne) {
            s = gal_load(elem, f);
            ns = nodes[f];
            near = !gal_is_far(o, s, no, ns, e, f);
        }
        const unsigned m = __ballot_sync(0xffffffffu, near);
        if (near) {
            const int at = pos + __popc(m & ((1u << lane) - 1u));
            col[at] = f;
            route[at] = gal_route(o, s, no, ns, e, f);
        }
        pos += __popc(m);
    }
}

// ------------------------------------------------------------------ Hankel functions
// (j/4) H0^(2)(x) and (j/4) k H1^(2)(x) for real x > 0.
//   x >= GAL_X_ASYM: H_nu^(2)(x) = sqrt(2/(pi x)) (P_nu - j Q_nu) e^{-j(x - nu pi/2 - pi/4)},
//   P_nu = sum_m (-1)^m a_2m(nu) x^-2m, Q_nu = sum_m (-1)^m a_2m+1(nu) x^-2m-1 (DLMF 10.17.3),
//   16 terms: the first omitted term is below 3e-16 of the sum at x = 25;
//   below: CUDA's double-precision j0, y0, j1, y1.
// Asymptotic branch with the first TERMS coefficients (TERMS even).
template <int TERMS>
__device__ __forceinline__ void gal_hankel_asym(double x, double k, double2 &g, double2 &hk) {
    const double inv = 1.0 / x;
    const double inv2 = inv * inv;
    // Horner in inv2 from the highest even / odd coefficient down
    double p0 = 0.0, q0 = 0.0, p1 = 0.0, q1 = 0.0;
#pragma unroll
    for (int m = TERMS / 2 - 1; m >= 0; --m) {
        const double sg = (m & 1) ? -1.0 : 1.0;
        p0 = fma(p0, inv2, sg * c_gal_a0[2 * m]);
        q0 = fma(q0, inv2, sg * c_gal_a0[2 * m + 1]);
        p1 = fma(p1, inv2, sg * c_gal_a1[2 * m]);
        q1 = fma(q1, inv2, sg * c_gal_a1[2 * m + 1]);
    }
    q0 *= inv;
    q1 *= inv;
    double sx, cx;
    sincos(x, &sx, &cx);
    // C = sqrt(2/(pi x)) e^{-j(x - pi/4)}, e^{-j(x - pi/4)} = ((c + s) - j (s - c)) / sqrt(2)
    const double amp = sqrt(inv * (1.0 / GRIM_PI));  // sqrt(2/(pi x)) / sqrt(2)
    const double cr = amp * (cx + sx), ci = -amp * (sx - cx);
    // g = (1/4)(Q0 + j P0) C ; hk = -(k/4)(P1 - j Q1) C
    g = make_double2(0.25 * (q0 * cr - p0 * ci), 0.25 * (q0 * ci + p0 * cr));
    const double kq = -0.25 * k;
    hk = make_double2(kq * (p1 * cr + q1 * ci), kq * (p1 * ci - q1 * cr));
}

// G and its normal-derivative factor at x = k r.  Above GAL_X_ASYM the DLMF 10.17 expansion,
// with as many terms as the argument needs for double precision (measured against SciPy's
// Hankel functions, worst of orders 0 and 1: 16 terms 2.8e-15 at x = 25; 12 terms 3e-15 at
// x = 35; 8 terms 8.5e-15 at x = 80, where the phase rounding already dominates); below it
// CUDA's j0 / y0 / j1 / y1.
__device__ __forceinline__ void gal_hankel(double x, double k, double2 &g, double2 &hk) {
    if (x >= 80.0) {
        gal_hankel_asym<8>(x, k, g, hk);
    } else if (x >= 35.0) {
        gal_hankel_asym<12>(x, k, g, hk);
    } else if (x >= GAL_X_ASYM) {
        gal_hankel_asym<GAL_ASYM64_TERMS>(x, k, g, hk);
    } else {
        const double j0v = j0(x), y0v = y0(x), j1v = j1(x), y1v = y1(x);
        // (j/4)(J0 - j Y0) = (Y0 + j J0)/4 ; (j/4) k (J1 - j Y1) = (k/4)(Y1 + j J1)
        g = make_double2(0.25 * y0v, 0.25 * j0v);
        hk = make_double2(0.25 * k * y1v, 0.25 * k * j1v);
    }
}

// Near-pair kernel values: r floored at GAL_EPS and k r at 1e-12 (the reference's floors).
__device__ __forceinline__ void gal_hankel_near(double r, double k, double2 &g, double2 &hk) {
    double x = k * fmax(r, GAL_EPS);
    if (fabs(x) <= 1e-12) x = 1e-12;
    const double j0v = j0(x), y0v = y0(x), j1v = j1(x), y1v = y1(x);
    g = make_double2(0.25 * y0v, 0.25 * j0v);
    hk = make_double2(0.25 * k * y1v, 0.25 * k * j1v);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// 2 x 2 complex blocks as 8 doubles: (re, im) of entry a*2+b.
struct GalBlk {
    double v[8];
};
__device__ __forceinline__ void gal_zero(GalBlk &b) {
#pragma unroll
    for (int i = 0; i < 8; ++i) b.v[i] = 0.0;
}
__device__ __forceinline__ void gal_warp_reduce(GalBlk &b) {
#pragma unroll
    for (int i = 0; i < 8; ++i) b.v[i] = warp_sum(b.v[i]);
}
__device__ __forceinline__ double gal_fro(const GalBlk &b) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += b.v[i] * b.v[i];
    return sqrt(s);
}

// Accumulate w * kern * phi_a(xo) * phi_b(xs) into blk.
__device__ __forceinline__ void gal_acc(GalBlk &blk, double w, double2 kern, double xo, double xs) {
    const double bo[2] = {1.0 - xo, xo}, bs[2] = {1.0 - xs, xs};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double c = w * bo[a] * bs[b];
            blk.v[2 * (2 * a + b)] = fma(c, kern.x, blk.v[2 * (2 * a + b)]);
            blk.v[2 * (2 * a + b) + 1] = fma(c, kern.y, blk.v[2 * (2 * a + b) + 1]);
        }
}

// ------------------------------------------------------------------ near rules (one warp each)
// Tensor rule of q x q Gauss points over the sub-intervals [oa, ob] x [sa, sb] of the two
// elements (parent parameters), in the parent hat bases; S and K' (observation normal),
// summed over the warp (every lane returns the totals).
__device__ void gal_box_warp(const GalElem &o, const GalElem &s, double k, double oa, double ob, double sa, double sb,
                             int q, GalBlk &S, GalBlk &K) {
    const int lane = threadIdx.x & 31;
    gal_zero(S);
    gal_zero(K);
    const double ho = fmax(ob - oa, 0.0), hs = fmax(sb - sa, 0.0);
    const double lo = o.len * ho, ls = s.len * hs;
    if (!(lo > 0.0) || !(ls > 0.0)) return;
    for (int idx = lane; idx < q * q; idx += 32) {
        const int i = idx / q, j = idx - i * q;
        double ti, wi, tj, wj;
        gal_gauss(q, i, ti, wi);
        gal_gauss(q, j, tj, wj);
        const double xo = oa + ho * ti, xs = sa + hs * tj;
        const double rx = (o.ax + xo * (o.bx - o.ax)) - (s.ax + xs * (s.bx - s.ax));
        const double ry = (o.ay + xo * (o.by - o.ay)) - (s.ay + xs * (s.by - s.ay));
        const double r = sqrt(rx * rx + ry * ry);
        double2 g, hk;
        gal_hankel_near(r, k, g, hk);
        const double w = wi * wj;
        gal_acc(S, w, g, xo, xs);
        if (r > GAL_EPS) {
            const double proj = -(rx * o.nx + ry * o.ny) / fmax(r, GAL_EPS);
            gal_acc(K, w, make_double2(hk.x * proj, hk.y * proj), xo, xs);
        }
    }
    gal_warp_reduce(S);
    gal_warp_reduce(K);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        S.v[i] *= lo * ls;
        K.v[i] *= lo * ls;
    }
}

// Graded corner rule of two elements sharing a node (obs_start / src_start: the shared
// node is that element's start point).  S and K' (observation normal).
__device__ void gal_touch_warp(const GalElem &o, const GalElem &s, bool obs_start, bool src_start, double k,
                               GalBlk &S, GalBlk &K) {
    const int lane = threadIdx.x & 31;
    gal_zero(S);
    gal_zero(K);
    const double cox = obs_start ? o.ax : o.bx, coy = obs_start ? o.ay : o.by;
    const double csx = src_start ? s.ax : s.bx, csy = src_start ? s.ay : s.by;
    const double dox = obs_start ? o.bx - o.ax : o.ax - o.bx, doy = obs_start ? o.by - o.ay : o.ay - o.by;
    const double dsx = src_start ? s.bx - s.ax : s.ax - s.bx, dsy = src_start ? s.by - s.ay : s.ay - s.by;
    double ox = cox - csx, oy = coy - csy;
    const double tiny = 64.0 * 2.220446049250313e-16 *
                        fmax(fmax(hypot(cox, coy), hypot(csx, csy)), fmax(o.len, s.len));
    if (hypot(ox, oy) <= tiny) ox = oy = 0.0;
    const int n = GAL_TOUCH_ORDER;
    for (int idx = lane; idx < 2 * n * n; idx += 32) {
        const int tri = idx / (n * n), rem = idx - tri * n * n;
        const int i = rem / n, j = rem - i * n;
        double ti, wi, tj, wj;
        gal_gauss(n, i, ti, wi);
        gal_gauss(n, j, tj, wj);
        const double t2 = ti * ti, u = t2 * t2;
        const double w = 4.0 * u * ti * ti * ti * wi * wj;
        const double x = tri == 0 ? u : u * tj;
        const double y = tri == 0 ? u * tj : u;
        const double rx = ox + x * dox - y * dsx, ry = oy + x * doy - y * dsy;
        const double xo = obs_start ? x : 1.0 - x;
        const double xs = src_start ? y : 1.0 - y;
        const double r = hypot(rx, ry);
        double2 g, hk;
        gal_hankel_near(r, k, g, hk);
        gal_acc(S, w, g, xo, xs);
        if (r > GAL_EPS) {
            const double proj = -(rx * o.nx + ry * o.ny) / r;
            gal_acc(K, w, make_double2(hk.x * proj, hk.y * proj), xo, xs);
        }
    }
    gal_warp_reduce(S);
    gal_warp_reduce(K);
    const double sc = o.len * s.len;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        S.v[i] *= sc;
        K.v[i] *= sc;
    }
}

// Single-layer block of the sub-interval [a, b] of a straight element by the small-argument
// series (parent basis); false where |k l| is outside (1e-30, 8] or the series fails.
__device__ bool gal_self_series(double length, double k, double a, double b, GalBlk &out) {
    gal_zero(out);
    const double ell = length * (b - a);
    if (ell <= 0.0) return true;
    const double z = k * ell;
    if (fabs(z) > GAL_SERIES_LIMIT || fabs(z) <= 1e-30) return false;
    // C_diag(u) = 2/3 - u + u^3/3, C_off(u) = 1/3 - u^3/3 ; moments int u^p = 1/(p+1),
    // int u^p ln u = -1/(p+1)^2 of c(u) u^(2m)
    const double cd[4] = {2.0 / 3.0, -1.0, 0.0, 1.0 / 3.0}, co[4] = {1.0 / 3.0, 0.0, 0.0, -1.0 / 3.0};
    const double c = 2.0 / GRIM_PI;
    const double shift = log(0.5 * z) + GRIM_EULER_GAMMA;
    const double quarter = 0.25 * z * z;
    double dre = 0.0, dim = 0.0, ore = 0.0, oim = 0.0;
    double term = 1.0, harmonic = 0.0;
    int m = 0;
    while (true) {
        double pd = 0.0, ld = 0.0, po = 0.0, lo = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double d1 = 1.0 / (2 * m + q + 1);
            pd += cd[q] * d1;
            ld -= cd[q] * d1 * d1;
            po += co[q] * d1;
            lo -= co[q] * d1 * d1;
        }
        // factor = term (1 - j c (shift - harmonic)); total += factor plain - j c term logged
        const double fi = -term * c * (shift - harmonic);
        dre += term * pd;
        dim += fi * pd - c * term * ld;
        ore += term * po;
        oim += fi * po - c * term * lo;
        m += 1;
        term *= -quarter / ((double)m * (double)m);
        harmonic += 1.0 / m;
        if (m > 60) return false;
        if (fabs(term) < 1e-18 * fmax(1.0, hypot(dre, dim))) break;
    }
    // block = (j/4) ell^2 [[d, o], [o, d]]
    const double sc = 0.25 * ell * ell;
    const double2 dg = make_double2(-sc * dim, sc * dre), od = make_double2(-sc * oim, sc * ore);
    if (a == 0.0 && b == 1.0) {
        out.v[0] = dg.x; out.v[1] = dg.y; out.v[2] = od.x; out.v[3] = od.y;
        out.v[4] = od.x; out.v[5] = od.y; out.v[6] = dg.x; out.v[7] = dg.y;
        return true;
    }
    // T B T^T with T = [[1 - a, 1 - b], [a, b]]
    const double T[2][2] = {{1.0 - a, 1.0 - b}, {a, b}};
    const double2 B[2][2] = {{dg, od}, {od, dg}};
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            double re = 0.0, im = 0.0;
#pragma unroll
            for (int p = 0; p < 2; ++p)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const double t = T[i][p] * T[j][q];
                    re += t * B[p][q].x;
                    im += t * B[p][q].y;
                }
            out.v[2 * (2 * i + j)] = re;
            out.v[2 * (2 * i + j) + 1] = im;
        }
    return true;
}

// Self block of an electrically long element (|k L| > 8): m sub-intervals with k L / m <= 2,
// each by the series, neighbouring sub-intervals by the graded corner rule, separated ones
// by the 16-point tensor rule, all in the parent basis (one warp).
__device__ bool gal_self_composite(double length, double k, GalBlk &out) {
    const int lane = threadIdx.x & 31;
    const double kl = fabs(k) * length;
    int m = max(2, (int)ceil(kl / GAL_SUB_KL));
    if (m > 256) m = max(256, (int)ceil(kl / GAL_SERIES_LIMIT));
    const double h = 1.0 / m;
    gal_zero(out);
    bool ok = true;
    for (int i = lane; i < m; i += 32) {
        GalBlk b;
        ok &= gal_self_series(length, k, i * h, (i + 1) * h, b);
#pragma unroll
        for (int v = 0; v < 8; ++v) out.v[v] += b.v[v];
    }
    ok = __all_sync(0xffffffffu, ok);
    const double eh = length * h;
    // neighbouring sub-intervals meeting at s = (i + 1) h, both sides
    const int n = GAL_TOUCH_ORDER;
    for (int idx = lane; idx < 2 * n * n * 2 * (m - 1); idx += 32) {
        const int joint = idx / (4 * n * n), rem0 = idx - joint * 4 * n * n;
        const int side = rem0 / (2 * n * n), rem = rem0 - side * 2 * n * n;
        const int tri = rem / (n * n), r2 = rem - tri * n * n;
        const int i = r2 / n, j = r2 - i * n;
        double ti, wi, tj, wj;
        gal_gauss(n, i, ti, wi);
        gal_gauss(n, j, tj, wj);
        const double t2 = ti * ti, u = t2 * t2;
        const double w = 4.0 * u * ti * ti * ti * wi * wj;
        const double x = tri == 0 ? u : u * tj;
        const double y = tri == 0 ? u * tj : u;
        const double sgn = side == 0 ? -1.0 : 1.0;
        const double jx = (joint + 1.0) * h;
        const double xo = jx + sgn * h * x, xs = jx - sgn * h * y;
        double2 g, hk;
        gal_hankel_near(eh * (x + y), k, g, hk);
        gal_acc(out, w * eh * eh, g, xo, xs);
    }
    // separated sub-intervals (offset d >= 2): the kernel depends on the offset only
    const int q = GAL_BOX_ORDER;
    for (int idx = lane; idx < (m - 2) * q * q; idx += 32) {
        const int d = 2 + idx / (q * q), rem = idx % (q * q);
        const int p = rem / q, qq = rem - p * q;
        double tp, wp, tq, wq;
        gal_gauss(q, p, tp, wp);
        gal_gauss(q, qq, tq, wq);
        double2 g, hk;
        gal_hankel_near(eh * (d + tq - tp), k, g, hk);
        const double w = wp * wq * eh * eh;
        for (int first = 0; first < m - d; ++first) {
            const double lower = (first + tp) * h, upper = (first + d + tq) * h;
            gal_acc(out, w, g, lower, upper);
            gal_acc(out, w, g, upper, lower);
        }
    }
    gal_warp_reduce(out);
    return ok;
}

// Close separated pairs (the adaptive route), one CTA of GAL_ADAPT_WARPS warps per pair:
// every box is compared with its four-way bisection (16-point tensor rule on each), and
// only the children whose parent missed the tolerance are refined further, to at most
// GAL_ADAPT_DEPTH levels (twod/operators.py:1172 _integrate_linear_pair_adaptive_sk).
// The reference walks the tree depth first; here the boxes still to refine sit on a stack
// in global memory (GAL_ADAPT_GCAP per pair) and each round takes up to GAL_ADAPT_BATCH of
// them from its top, the warps evaluating all their children side by side.  Each box's
// decision depends only on itself and its children, so both visit the same boxes; only
// the order of the final sum differs.  A box unconverged at the last level, or a stack
// overflow, sets err_flag (the reference raises for the first).
#define GAL_ADAPT_WARPS 16
#define GAL_ADAPT_BATCH 64
#define GAL_ADAPT_GCAP 4096

struct GalBox {
    double oa, ob, sa, sb;
    GalBlk cs, ck;
    int depth, pad;
};

__device__ __forceinline__ void gal_child(const GalBox &b, int c, double &oa, double &ob, double &sa, double &sb) {
    const double om = 0.5 * (b.oa + b.ob), sm = 0.5 * (b.sa + b.sb);
    oa = c < 2 ? b.oa : om;
    ob = c < 2 ? om : b.ob;
    sa = (c & 1) ? sm : b.sa;
    sb = (c & 1) ? b.sb : sm;
}

__global__ void __launch_bounds__(GAL_ADAPT_WARPS * 32)
k_gal_adapt(int ne, int nadapt, const int *__restrict__ adapt_idx, const double *__restrict__ elem,
            const int *__restrict__ row_off, const int *__restrict__ col, double k, GalBox *__restrict__ stacks,
            double2 *__restrict__ NBK, int *__restrict__ err_flag) {
    extern __shared__ __align__(16) unsigned char gal_smem[];
    GalBox *cur = reinterpret_cast<GalBox *>(gal_smem);                    // this round's boxes
    GalBlk *kid = reinterpret_cast<GalBlk *>(cur + GAL_ADAPT_BATCH);       // 2 per child: S, K'
    __shared__ int s_top, s_fail, s_push[GAL_ADAPT_BATCH + 1];
    __shared__ unsigned char conv[GAL_ADAPT_BATCH];
    __shared__ double tot[16];
    if (blockIdx.x >= nadapt) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    GalBox *stack = stacks + (size_t)blockIdx.x * GAL_ADAPT_GCAP;
    const int idx = adapt_idx[blockIdx.x];
    int lo = 0, hi = ne;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (row_off[mid] <= idx) lo = mid;
        else hi = mid;
    }
    const GalElem o = gal_load(elem, lo), s = gal_load(elem, col[idx]);
    const double floor_ = 2.220446049250313e-16 * fmax(1.0, o.len * s.len);
    if (warp == 0) {
        GalBlk cs, ck;
        gal_box_warp(o, s, k, 0.0, 1.0, 0.0, 1.0, GAL_BOX_ORDER, cs, ck);
        if (lane == 0) {
            GalBox &b = stack[0];
            b.oa = 0.0; b.ob = 1.0; b.sa = 0.0; b.sb = 1.0;
            b.cs = cs; b.ck = ck; b.depth = 0;
            s_top = 1;
            s_fail = 0;
        }
    }
    if (tid < 16) tot[tid] = 0.0;
    __syncthreads();
    while (s_top > 0) {
        const int top = s_top;
        const int nb = min(top, GAL_ADAPT_BATCH), base = top - nb;
        for (int i = tid; i < nb; i += blockDim.x) cur[i] = stack[base + i];
        __syncthreads();
        for (int ci = warp; ci < 4 * nb; ci += GAL_ADAPT_WARPS) {
            double oa, ob, sa, sb;
            gal_child(cur[ci >> 2], ci & 3, oa, ob, sa, sb);
            GalBlk ks, kk;
            gal_box_warp(o, s, k, oa, ob, sa, sb, GAL_BOX_ORDER, ks, kk);
            if (lane == 0) {
                kid[2 * ci] = ks;
                kid[2 * ci + 1] = kk;
            }
        }
        __syncthreads();
        for (int i = tid; i < nb; i += blockDim.x) {
            double ns = 0.0, nk = 0.0;
            GalBlk ds, dk;
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                ds.v[v] = -cur[i].cs.v[v];
                dk.v[v] = -cur[i].ck.v[v];
            }
            for (int c = 0; c < 4; ++c) {
                const GalBlk &a = kid[2 * (4 * i + c)], &b = kid[2 * (4 * i + c) + 1];
#pragma unroll
                for (int v = 0; v < 8; ++v) {
                    ds.v[v] += a.v[v];
                    dk.v[v] += b.v[v];
                }
                ns += gal_fro(a);
                nk += gal_fro(b);
            }
            const double err = fmax(gal_fro(ds) / fmax(ns, floor_), gal_fro(dk) / fmax(nk, floor_));
            conv[i] = err <= GAL_ADAPT_RTOL ? 1 : 0;
        }
        __syncthreads();
        if (tid == 0) {
            // converged boxes (or boxes at the last level, or with no stack room) add their
            // children in a fixed order; the others push theirs
            int pushed = base;
            for (int i = 0; i < nb; ++i) {
                s_push[i] = -1;
                const bool stop = conv[i] || cur[i].depth >= GAL_ADAPT_DEPTH || pushed + 4 > GAL_ADAPT_GCAP;
                if (stop) {
                    if (!conv[i]) s_fail = 1;
                    for (int c = 0; c < 4; ++c)
#pragma unroll
                        for (int v = 0; v < 8; ++v) {
                            tot[v] += kid[2 * (4 * i + c)].v[v];
                            tot[8 + v] += kid[2 * (4 * i + c) + 1].v[v];
                        }
                } else {
                    s_push[i] = pushed;
                    pushed += 4;
                }
            }
            s_top = pushed;
        }
        __syncthreads();
        // child 0 ends on top of each pushed group, so it is taken first
        for (int e = tid; e < 4 * nb; e += blockDim.x) {
            const int i = e >> 2, c = e & 3;
            if (s_push[i] < 0) continue;
            GalBox &d = stack[s_push[i] + 3 - c];
            gal_child(cur[i], c, d.oa, d.ob, d.sa, d.sb);
            d.cs = kid[2 * e];
            d.ck = kid[2 * e + 1];
            d.depth = cur[i].depth + 1;
        }
        __syncthreads();
    }
    if (tid == 0 && s_fail) atomicExch(err_flag, 1);
    if (tid < 8) {
        double2 *out = NBK + 8 * (size_t)idx;
        if (tid < 4) out[tid] = make_double2(tot[2 * tid], tot[2 * tid + 1]);
        else out[tid] = make_double2(tot[8 + 2 * (tid - 4)], tot[8 + 2 * (tid - 4) + 1]);
    }
}

#define GAL_ADAPT_SMEM ((size_t)GAL_ADAPT_BATCH * sizeof(GalBox) + (size_t)8 * GAL_ADAPT_BATCH * sizeof(GalBlk))

// S and K' of every near pair: NBK[idx] = 8 double2 (S entries a*2+b, then K').  One warp per
// pair; err_flag set when an adaptive pair did not converge or a self series failed.
__global__ void __launch_bounds__(GAL_NEAR_WARPS * 32)
k_gal_near(int ne, int nnz, const double *__restrict__ elem, const int2 *__restrict__ nodes,
           const int *__restrict__ row_off, const int *__restrict__ col, const int *__restrict__ route, double k,
           double2 *__restrict__ NBK, int *__restrict__ err_flag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int idx = blockIdx.x * GAL_NEAR_WARPS + warp;
    if (idx >= nnz) return;
    // row of idx by binary search in row_off
    int lo = 0, hi = ne;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (row_off[mid] <= idx) lo = mid;
        else hi = mid;
    }
    const int e = lo, f = col[idx], rt = route[idx];
    const GalElem o = gal_load(elem, e), s = gal_load(elem, f);
    GalBlk S, K;
    bool ok = true;
    if (rt == GAL_ROUTE_SELF) {
        gal_zero(K);
        if (fabs(k) * o.len > GAL_SERIES_LIMIT) ok = gal_self_composite(o.len, k, S);
        else ok = gal_self_series(o.len, k, 0.0, 1.0, S);
    } else if (rt == GAL_ROUTE_TOUCH) {
        const int2 no = nodes[e], ns = nodes[f];
        const bool obs_start = no.x == ns.x || no.x == ns.y;
        const bool src_start = ns.x == no.x || ns.x == no.y;
        gal_touch_warp(o, s, obs_start, src_start, k, S, K);
    } else if (rt == GAL_ROUTE_ADAPT) {
        return;  // k_gal_adapt
    } else {
        gal_box_warp(o, s, k, 0.0, 1.0, 0.0, 1.0, GAL_BOX_ORDER, S, K);
    }
    if (!ok && lane == 0) atomicExch(err_flag, 1);
    if (lane < 8) {
        double2 *out = NBK + 8 * (size_t)idx;
        if (lane < 4) out[lane] = make_double2(S.v[2 * lane], S.v[2 * lane + 1]);
        else out[lane] = make_double2(K.v[2 * (lane - 4)], K.v[2 * (lane - 4) + 1]);
    }
}

// Maue hypersingular block from the single-layer block.
__device__ __forceinline__ void gal_maue(const double2 S[4], double k, double ndn, double lo, double ls, double2 W[4]) {
    const double tr = (S[0].x + S[1].x) + (S[2].x + S[3].x), ti = (S[0].y + S[1].y) + (S[2].y + S[3].y);
    const double den = fmax(lo * ls, GAL_EPS * GAL_EPS);
    const double qr = tr / den, qi = ti / den;
    const double c = -(k * k) * ndn;
    const double sg[4] = {1.0, -1.0, -1.0, 1.0};
#pragma unroll
    for (int i = 0; i < 4; ++i) W[i] = make_double2(c * S[i].x + sg[i] * qr, c * S[i].y + sg[i] * qi);
}

// Routed element blocks of the near pairs (and the mass on self pairs) into E (layout:
// block (row e, col f) at E[(f * ne + e) * 4 + a * 2 + b]).
template <int POL, typename C>
__global__ void k_gal_near_route(int ne, int nnz, const double *__restrict__ elem, const int *__restrict__ row_off,
                                 const int *__restrict__ col, const double2 *__restrict__ NBK, double k,
                                 C *__restrict__ E) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nnz) return;
    int lo = 0, hi = ne;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (row_off[mid] <= idx) lo = mid;
        else hi = mid;
    }
    const int e = lo, f = col[idx];
    const double2 *nb = NBK + 8 * (size_t)idx;
    double2 S[4], out[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) S[i] = nb[i];
    // gamma = 1/(j k) = -j/k
    const double gi = -1.0 / k;
    const GalElem o = gal_load(elem, e), s = gal_load(elem, f);
    if (POL == GRIM_POL_TM) {
        // D_ef[a][b] = K'_fe[b][a]: the (f, e) pair's block, found in row f
        int a0 = row_off[f], a1 = row_off[f + 1];
        while (a1 - a0 > 1) {
            const int mid = (a0 + a1) >> 1;
            if (col[mid] <= e) a0 = mid;
            else a1 = mid;
        }
        const double2 *kt = NBK + 8 * (size_t)a0 + 4;
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const double2 d = kt[2 * b + a];
                // S + gamma D, gamma D = (-j/k) d = (d.y/k, -d.x/k)
                out[2 * a + b] = make_double2(S[2 * a + b].x - gi * d.y, S[2 * a + b].y + gi * d.x);
            }
        if (e == f) {
            // + gamma M/2, M = L [[1/3, 1/6], [1/6, 1/3]]: gamma M/2 is imaginary
            const double m0 = o.len / 3.0, m1 = o.len / 6.0;
            out[0].y += 0.5 * gi * m0;
            out[1].y += 0.5 * gi * m1;
            out[2].y += 0.5 * gi * m1;
            out[3].y += 0.5 * gi * m0;
        }
    } else {
        double2 W[4];
        gal_maue(S, k, o.nx * s.nx + o.ny * s.ny, o.len, s.len, W);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double2 kp = nb[4 + i];
            // K' - gamma W, gamma W = (-j/k) W = (W.y/k, -W.x/k)
            out[i] = make_double2(kp.x + gi * W[i].y, kp.y - gi * W[i].x);
        }
        if (e == f) {
            const double m0 = o.len / 3.0, m1 = o.len / 6.0;
            out[0].x -= 0.5 * m0;
            out[1].x -= 0.5 * m1;
            out[2].x -= 0.5 * m1;
            out[3].x -= 0.5 * m0;
        }
    }
    C *dst = E + ((size_t)f * ne + e) * 4;
#pragma unroll
    for (int i = 0; i < 4; ++i) dst[i] = conv<C>(out[i]);
}

// Calibrated far order of a tile (linear elements, real k): kl_max = |k| max(L) over the
// tile's elements, ratio_min the smallest centre-distance ratio of its far pairs.
__device__ __forceinline__ int gal_far_order(double kl_max, double ratio_min, int cap) {
    if (!(ratio_min >= GAL_FAR_RATIO)) return cap;
    const double bounds[4] = {0.15, 0.50, 1.50, 3.00};
    const int orders[4][3] = {{7, 6, 5}, {7, 6, 5}, {7, 6, 6}, {8, 8, 8}};
    for (int i = 0; i < 4; ++i)
        if (kl_max <= bounds[i]) {
            const int o = ratio_min < 5.0 ? orders[i][0] : (ratio_min < 10.0 ? orders[i][1] : orders[i][2]);
            return max(2, min(cap, o));
        }
    return cap;
}

#define GAL_MAX_Q 16

// Far pairs of one 32 x 32 tile of the upper tile triangle (rows ti <= cols tj); pairs
// e < f only on diagonal tiles.  One set of Hankel evaluations per pair gives both
// orientations: E[e][f] and E[f][e].  min_order: the floor on the tile order (the TE rows'
// W rule: 8, or 16 outside its calibration; 0 for TM).
// Two CTAs per SM (at most 128 registers a thread): 16 warps hide the FP64 latency of the
// Hankel evaluations better than 8 (the accumulators of the pair spill a few words).
template <int POL, typename C>
__global__ void __launch_bounds__(GAL_FAR_THREADS, 2)
k_gal_far(int ne, const double *__restrict__ elem, const int2 *__restrict__ nodes, double k, int min_order,
          C *__restrict__ E) {
    const int ti = blockIdx.y, tj = blockIdx.x;
    if (ti > tj) return;
    __shared__ GalElem so[GAL_TILE], ss[GAL_TILE];
    __shared__ int2 sno[GAL_TILE], sns[GAL_TILE];
    __shared__ double red_r[GAL_FAR_THREADS / 32], red_l[GAL_FAR_THREADS / 32];
    __shared__ double qt[GAL_MAX_Q], qw[GAL_MAX_Q];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int e0 = ti * GAL_TILE, f0 = tj * GAL_TILE;
    if (tid < GAL_TILE) {
        const int e = min(e0 + tid, ne - 1), f = min(f0 + tid, ne - 1);
        so[tid] = gal_load(elem, e);
        ss[tid] = gal_load(elem, f);
        sno[tid] = nodes[e];
        sns[tid] = nodes[f];
    }
    __syncthreads();
    // tile order from its worst far pair
    double rmin = INFINITY, lmax = 0.0;
    for (int p = tid; p < GAL_TILE * GAL_TILE; p += GAL_FAR_THREADS) {
        const int le = p & (GAL_TILE - 1), lf = p >> 5;
        const int e = e0 + le, f = f0 + lf;
        if (e < ne && f < ne) {
            lmax = fmax(lmax, fmax(so[le].len, ss[lf].len));
            if (gal_is_far(so[le], ss[lf], sno[le], sns[lf], e, f)) rmin = fmin(rmin, gal_ratio(so[le], ss[lf]));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rmin = fmin(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
        lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    }
    if (lane == 0) {
        red_r[warp] = rmin;
        red_l[warp] = lmax;
    }
    __syncthreads();
    if (tid == 0) {
        double r = INFINITY, l = 0.0;
        for (int w = 0; w < GAL_FAR_THREADS / 32; ++w) {
            r = fmin(r, red_r[w]);
            l = fmax(l, red_l[w]);
        }
        red_r[0] = r;
        red_l[0] = l;
    }
    __syncthreads();
    if (!(red_r[0] < INFINITY)) return;  // no far pair in this tile
    const int q = min(GAL_MAX_Q, max(min_order, gal_far_order(fabs(k) * red_l[0], red_r[0], 8)));
    if (tid < q) gal_gauss(q, tid, qt[tid], qw[tid]);
    __syncthreads();
    const double gi = -1.0 / k;  // gamma = 1/(j k) = -j/k
    for (int p = tid; p < GAL_TILE * GAL_TILE; p += GAL_FAR_THREADS) {
        const int le = p & (GAL_TILE - 1), lf = p >> 5;
        const int e = e0 + le, f = f0 + lf;
        if (e >= ne || f >= ne) continue;
        if (ti == tj && e >= f) continue;
        const GalElem o = so[le], s = ss[lf];
        if (!gal_is_far(o, s, sno[le], sns[lf], e, f)) continue;
        double S[8], A[8], B[8];  // S; sum h (r.n_s)/r ; sum h (r.n_o)/r  (entries a*2+b, re/im)
#pragma unroll
        for (int i = 0; i < 8; ++i) S[i] = A[i] = B[i] = 0.0;
        const double odx = o.bx - o.ax, ody = o.by - o.ay, sdx = s.bx - s.ax, sdy = s.by - s.ay;
        for (int ip = 0; ip < q; ++ip) {
            const double tp = qt[ip];
            const double xpx = o.ax + tp * odx, xpy = o.ay + tp * ody;
            double rs0x = 0, rs0y = 0, rs1x = 0, rs1y = 0, ra0x = 0, ra0y = 0, ra1x = 0, ra1y = 0;
            double rb0x = 0, rb0y = 0, rb1x = 0, rb1y = 0;
            for (int iq = 0; iq < q; ++iq) {
                const double tq = qt[iq], wq = qw[iq];
                const double rx = xpx - (s.ax + tq * sdx), ry = xpy - (s.ay + tq * sdy);
                const double r2 = rx * rx + ry * ry;
                const double ir = rsqrt(r2);
                const double r = r2 * ir;
                double2 g, hk;
                gal_hankel(k * r, k, g, hk);
                const double pa = (rx * s.nx + ry * s.ny) * ir, pb = (rx * o.nx + ry * o.ny) * ir;
                const double w1 = wq * tq, w0 = wq - w1;
                rs0x = fma(w0, g.x, rs0x); rs0y = fma(w0, g.y, rs0y);
                rs1x = fma(w1, g.x, rs1x); rs1y = fma(w1, g.y, rs1y);
                const double hax = hk.x * pa, hay = hk.y * pa, hbx = hk.x * pb, hby = hk.y * pb;
                ra0x = fma(w0, hax, ra0x); ra0y = fma(w0, hay, ra0y);
                ra1x = fma(w1, hax, ra1x); ra1y = fma(w1, hay, ra1y);
                rb0x = fma(w0, hbx, rb0x); rb0y = fma(w0, hby, rb0y);
                rb1x = fma(w1, hbx, rb1x); rb1y = fma(w1, hby, rb1y);
            }
            const double wp = qw[ip];
            const double v1 = wp * tp, v0 = wp - v1;
            S[0] = fma(v0, rs0x, S[0]); S[1] = fma(v0, rs0y, S[1]); S[2] = fma(v0, rs1x, S[2]); S[3] = fma(v0, rs1y, S[3]);
            S[4] = fma(v1, rs0x, S[4]); S[5] = fma(v1, rs0y, S[5]); S[6] = fma(v1, rs1x, S[6]); S[7] = fma(v1, rs1y, S[7]);
            A[0] = fma(v0, ra0x, A[0]); A[1] = fma(v0, ra0y, A[1]); A[2] = fma(v0, ra1x, A[2]); A[3] = fma(v0, ra1y, A[3]);
            A[4] = fma(v1, ra0x, A[4]); A[5] = fma(v1, ra0y, A[5]); A[6] = fma(v1, ra1x, A[6]); A[7] = fma(v1, ra1y, A[7]);
            B[0] = fma(v0, rb0x, B[0]); B[1] = fma(v0, rb0y, B[1]); B[2] = fma(v0, rb1x, B[2]); B[3] = fma(v0, rb1y, B[3]);
            B[4] = fma(v1, rb0x, B[4]); B[5] = fma(v1, rb0y, B[5]); B[6] = fma(v1, rb1x, B[6]); B[7] = fma(v1, rb1y, B[7]);
        }
        const double sc = o.len * s.len;
        double2 Sb[4], Ab[4], Bb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Sb[i] = make_double2(sc * S[2 * i], sc * S[2 * i + 1]);
            Ab[i] = make_double2(sc * A[2 * i], sc * A[2 * i + 1]);
            Bb[i] = make_double2(sc * B[2 * i], sc * B[2 * i + 1]);
        }
        double2 ef[4], fe[4];  // E[e][f][a][b] ; E[f][e][b][a] stored at index a*2+b
        if (POL == GRIM_POL_TM) {
            // E_ef = S + gamma D_ef, D_ef = A ; E_fe[b][a] = S[a][b] + gamma D_fe[b][a], D_fe[b][a] = -B[a][b]
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ef[i] = make_double2(Sb[i].x - gi * Ab[i].y, Sb[i].y + gi * Ab[i].x);
                fe[i] = make_double2(Sb[i].x + gi * Bb[i].y, Sb[i].y - gi * Bb[i].x);
            }
        } else {
            // E_ef = K'_ef - gamma W, K'_ef = -B ; E_fe[b][a] = K'_fe[b][a] - gamma W[a][b], K'_fe[b][a] = A[a][b]
            double2 W[4];
            gal_maue(Sb, k, o.nx * s.nx + o.ny * s.ny, o.len, s.len, W);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ef[i] = make_double2(-Bb[i].x + gi * W[i].y, -Bb[i].y - gi * W[i].x);
                fe[i] = make_double2(Ab[i].x + gi * W[i].y, Ab[i].y - gi * W[i].x);
            }
        }
        C *d1 = E + ((size_t)f * ne + e) * 4;
        C *d2 = E + ((size_t)e * ne + f) * 4;
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                d1[2 * a + b] = conv<C>(ef[2 * a + b]);
                d2[2 * b + a] = conv<C>(fe[2 * a + b]);
            }
    }
}

// Node matrix: Z[i][j] = sum of E[e][f][a][b] over the elements e with node a = i and f with
// node b = j (start_of / end_of: the element that starts / ends at each node, -1 for none).
template <typename C>
__global__ void k_gal_gather(int ne, int n, const int *__restrict__ start_of, const int *__restrict__ end_of,
                             const C *__restrict__ E, C *__restrict__ Z, int64_t ldz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    const int si = start_of[i], ei = end_of[i], sj = start_of[j], ej = end_of[j];
    double re = 0.0, im = 0.0;
    auto add = [&](int e, int f, int a, int b) {
        if (e < 0 || f < 0) return;
        const C v = E[((size_t)f * ne + e) * 4 + 2 * a + b];
        re += (double)v.x;
        im += (double)v.y;
    };
    add(si, sj, 0, 0);
    add(si, ej, 0, 1);
    add(ei, sj, 1, 0);
    add(ei, ej, 1, 1);
    Z[(size_t)j * ldz + i] = conv<C>(make_double2(re, im));
}

// Galerkin plane-wave loads of node i for angle r (d = (cos phi, sin phi), u = e^{j k d.x}):
//   load_i    = sum over the elements at node i of L int phi_a(t) u(x(t)) dt
//   dn_load_i = the same with the factor j k (d . n)
// TM: B = -load ; TE: B = -dn_load.  8 Gauss points per element.
template <int POL, typename C>
__global__ void k_gal_rhs(int n, const double *__restrict__ elem, const int *__restrict__ start_of,
                          const int *__restrict__ end_of, int nang, const double *__restrict__ angles_deg, double k,
                          C *__restrict__ B, int64_t ldb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (i >= n) return;
    const double phi = angles_deg[r] * (GRIM_PI / 180.0);
    double dx, dy;
    sincos(phi, &dy, &dx);
    double re = 0.0, im = 0.0;
    for (int side = 0; side < 2; ++side) {
        const int e = side == 0 ? start_of[i] : end_of[i];
        if (e < 0) continue;
        const GalElem g = gal_load(elem, e);
        const double dn = dx * g.nx + dy * g.ny;
        double lr = 0.0, li = 0.0;
        for (int qi = 0; qi < GAL_LOAD_ORDER; ++qi) {
            double t, w;
            gal_gauss(GAL_LOAD_ORDER, qi, t, w);
            const double px = g.ax + t * (g.bx - g.ax), py = g.ay + t * (g.by - g.ay);
            double sp, cp;
            sincos(k * (dx * px + dy * py), &sp, &cp);
            const double sh = w * (side == 0 ? 1.0 - t : t);
            lr = fma(sh, cp, lr);
            li = fma(sh, sp, li);
        }
        lr *= g.len;
        li *= g.len;
        if (POL == GRIM_POL_TM) {
            re += lr;
            im += li;
        } else {
            // j k dn (lr + j li) = k dn (-li + j lr)
            re -= k * dn * li;
            im += k * dn * lr;
        }
    }
    B[(size_t)r * ldb + i] = conv<C>(make_double2(-re, -im));
}

// Monostatic far field of the combined density X (one column per angle):
//   amp = sum_e L_e int (phi_0 rho_n0 + phi_1 rho_n1) e^{j k d.x} (1 + gamma j k (d . n_e)),
// gamma = 1/(j k), so the factor is 1 + (d . n_e).  One CTA per angle, fixed-order reduction.
template <typename C>
__global__ void k_gal_farfield(int ne, const double *__restrict__ elem, const int2 *__restrict__ nodes, int nang,
                               const double *__restrict__ angles_deg, double k, const C *__restrict__ X, int64_t ldx,
                               double2 *__restrict__ amp) {
    __shared__ double sre[256], sim[256];
    const int r = blockIdx.x;
    const double phi = angles_deg[r] * (GRIM_PI / 180.0);
    double dx, dy;
    sincos(phi, &dy, &dx);
    double re = 0.0, im = 0.0;
    const C *x = X + (size_t)r * ldx;
    for (int e = threadIdx.x; e < ne; e += blockDim.x) {
        const GalElem g = gal_load(elem, e);
        const int2 nd = nodes[e];
        const double2 r0 = to_c64(x[nd.x]), r1 = to_c64(x[nd.y]);
        const double fac = 1.0 + (dx * g.nx + dy * g.ny);
        double ar = 0.0, ai = 0.0;
        for (int qi = 0; qi < GAL_LOAD_ORDER; ++qi) {
            double t, w;
            gal_gauss(GAL_LOAD_ORDER, qi, t, w);
            const double px = g.ax + t * (g.bx - g.ax), py = g.ay + t * (g.by - g.ay);
            double sp, cp;
            sincos(k * (dx * px + dy * py), &sp, &cp);
            const double dr = (1.0 - t) * r0.x + t * r1.x, di = (1.0 - t) * r0.y + t * r1.y;
            ar = fma(w, dr * cp - di * sp, ar);
            ai = fma(w, dr * sp + di * cp, ai);
        }
        re = fma(g.len * fac, ar, re);
        im = fma(g.len * fac, ai, im);
    }
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sre[threadIdx.x] += sre[threadIdx.x + s];
            sim[threadIdx.x] += sim[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) amp[r] = make_double2(sre[0], sim[0]);
}
