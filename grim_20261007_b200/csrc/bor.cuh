// Body-of-revolution PEC EFIE / MFIE / CFIE, per azimuthal mode.
//
// Stage 1  element-pair moments, mode-independent, for n = 0..mmax+1:
//   EFIE, from the modal Green's function G_n = int_{-pi}^{pi} e^{-jkR}/(4 pi R) cos(n xi) dxi:
//     A_ac  = sum T_a T_c rho rho' w w' G_n      DD_ac = sum D_a D_c w w' G_n
//     DT_ac = sum D_a T_c w w' G_n               TD_ac = sum T_a D_c w w' G_n
//     TT_ac = sum T_a T_c w w' G_n               (a, c in {0, 1}: the element's two tents)
//   MFIE (optional), from the four modal brackets K^n_uv = int F_uv(xi) e^{-j n xi} dxi
//   (uv = tt, tf, ft, ff; tt/ff even in xi, tf/ft odd):
//     B_uv,ac = sum T_a T_c rho rho' w w' K^n_uv
//   Layouts: mom[((e * ne + f) * (mmax + 2) + n) * 20 + slot],
//            momk[((e * ne + f) * (mmax + 2) + n) * 16 + 4 uv + 2 a + c], complex128.
//   The element pairs follow the reference's routing (bor/solver.py:1520-1580): far pairs
//   take 3 x 3 Gauss points and the uniform trapezoid rule in xi (k_bor_far, one CTA per
//   pair); near pairs take the host's point list -- graded cells for self / adjacent pairs
//   (bor/solver.py:718-806), a 12 x 12 Gauss rule for the others (:843) -- and a composite
//   rule on xi in [0, pi] using each integrand's parity (k_bor_near over work items of at
//   most BOR_NEAR_CHUNK point pairs, then k_bor_near_reduce in a fixed order).
// Stage 2  k_bor_assemble: the reduced mode-m matrix alpha C EFIE + (1 - alpha) eta0
//   ((1/2) M - K), C = j k eta 2 pi, from the moments of the <= 4 element pairs touching
//   each node pair, with the pole treatment (inactive pole phi components, |m| = 1 pole t
//   component tied to phi by j m sign(t_rho)).
// Stage 3  k_bor_excitation: reduced right-hand sides alpha <W, E_inc> + (1 - alpha) eta0
//   <W, n x H_inc> (VV, HH per aspect) or far-field weights, with the phi integrals in
//   closed form through J_m (CUDA's jn).
// Reference: bor/solver.py:1769-1827 (assemble_mode), :1962 (assemble_mfie_mode),
// :2048 (rhs_mfie_mode), :2369-2440 (pole reduction), :2558-2608 (rhs_vv_hh_batch /
// farfield_vv_hh_batch), :4285-4301 (CFIE), bor/kernels.py:896,996 (MFIE brackets).
#pragma once
#include "common.cuh"

#define BOR_FAR_ORDER 3
#define BOR_MAX_MODES 128
#define BOR_MAX_NXI 8192
#define BOR_SLOTS 20
#define BOR_KSLOTS 16
#define BOR_ALL_SLOTS (BOR_SLOTS + BOR_KSLOTS)
#define BOR_THREADS 256
#define BOR_FAR_CHUNK 256   // far-pair xi samples staged per pass
#define BOR_NEAR_CHUNK 64   // point pairs per near work item
#define BOR_XI_CORE 20      // Gauss points of the near rule's sinh core
#define BOR_XI_PANEL 16     // Gauss points per panel of the near rule

struct BorPt {
    double rho, z, w, T0, T1, D0, D1, tr, tz;
};

__device__ __forceinline__ BorPt bor_point(const double *nodes, int e, double s, double ws) {
    const double r0 = nodes[2 * e], z0 = nodes[2 * e + 1], r1 = nodes[2 * e + 2], z1 = nodes[2 * e + 3];
    const double dr = r1 - r0, dz = z1 - z0, L = sqrt(dr * dr + dz * dz);
    const double trho = dr / L;
    BorPt p;
    p.rho = r0 + s * dr;
    p.z = z0 + s * dz;
    p.w = ws * L;
    p.T0 = 1.0 - s;
    p.T1 = s;
    p.D0 = p.rho * (-1.0 / L) + p.T0 * trho;
    p.D1 = p.rho * (1.0 / L) + p.T1 * trho;
    p.tr = trho;
    p.tz = dz / L;
    return p;
}

// Far-pair xi sample count (multiple of 32, so that sin(x) = cos(x - pi/2) is a table shift).
__device__ __forceinline__ int bor_nxi(double k, double rp, double rq, double r0, int mmax) {
    const double c = sqrt(rp * rq);
    const double v = 1.5 * (2.0 * k * c + mmax + 2) + 40.0 * c / fmax(r0, 1e-300) + 16.0;
    int n = 32 * (int)ceil(v / 32.0);
    return n > BOR_MAX_NXI ? BOR_MAX_NXI : n;
}

// Gauss-Legendre nodes/weights (orders 1..32) from the 2-D fill's constant tables.
__device__ __forceinline__ void gl_node(int q, int i, double &x, double &w) {
    x = c_gl_x[q * (q - 1) / 2 + i];
    w = c_gl_w[q * (q - 1) / 2 + i];
}

// Geometry of one point pair shared by every xi sample.
struct BorPair {
    double k, rp, rq, dr, dz, d2, rr2;     // rr2 = 2 rho rho'
    double A, N, X, D, trp, tzp, trq, tzq;  // MFIE bracket invariants
};

__device__ __forceinline__ BorPair bor_pair(double k, const BorPt &p, const BorPt &q) {
    BorPair s;
    s.k = k;
    s.rp = p.rho;
    s.rq = q.rho;
    s.dr = p.rho - q.rho;
    s.dz = p.z - q.z;
    s.d2 = s.dr * s.dr + s.dz * s.dz;
    s.rr2 = 2.0 * p.rho * q.rho;
    s.trp = p.tr;
    s.tzp = p.tz;
    s.trq = q.tr;
    s.tzq = q.tz;
    s.X = p.tr * q.tz - p.tz * q.tr;
    s.D = p.tr * q.tr + p.tz * q.tz;
    s.A = p.tr * s.dr + p.tz * s.dz;
    s.N = -p.tz * s.dr + p.tr * s.dz;
    return s;
}

// One xi sample times weight wt: the Green's function g and (MFIE) the four brackets
// -p(R) [tt, tf, ft, ff] in the cancellation-free form (h = 1 - cos xi = 2 sin^2(xi/2)).
template <bool MFIE>
__device__ __forceinline__ void bor_sample(const BorPair &s, double shalf, double sx, double wt, double2 &g,
                                           double2 (&F)[4]) {
    const double h = 2.0 * shalf * shalf;
    const double R = sqrt(s.d2 + s.rr2 * h);
    double sk, ck;
    sincos(s.k * R, &sk, &ck);
    const double a = wt / (4.0 * GRIM_PI * R);
    g = make_double2(a * ck, -a * sk);
    if constexpr (MFIE) {
        const double kr = s.k * R;
        const double pre = a / (R * R);
        // -(1 + j kR) e^{-jkR} / (4 pi R^3) times the weight
        const double pr = -pre * (ck + kr * sk), pi = -pre * (kr * ck - sk);
        const double tt = (s.A * s.X - s.D * s.N) +
                          h * (s.A * s.tzp * s.trq + s.trp * s.rq * s.X + s.D * s.tzp * s.rq + s.trp * s.trq * s.N);
        const double tf = -sx * s.dz * (s.trp * s.trp + s.tzp * s.tzp);
        const double ft = sx * (s.rq * s.X + s.trq * s.N);
        const double ff = -s.tzp * s.rq * h - s.N * (1.0 - h);
        F[0] = make_double2(pr * tt, pi * tt);
        F[1] = make_double2(pr * tf, pi * tf);
        F[2] = make_double2(pr * ft, pi * ft);
        F[3] = make_double2(pr * ff, pi * ff);
    }
}

// The 36 per-point-pair factors multiplying G_n (slots 0..19) or K^n_uv (slots 20..35).
__device__ __forceinline__ double bor_factor(const BorPt &p, const BorPt &q, int slot) {
    const int ac = slot & 3, a = ac >> 1, c = ac & 1;
    const double Ta = a ? p.T1 : p.T0, Tc = c ? q.T1 : q.T0;
    const double Da = a ? p.D1 : p.D0, Dc = c ? q.D1 : q.D0;
    const double ww = p.w * q.w;
    if (slot >= BOR_SLOTS) return Ta * Tc * (p.rho * q.rho * ww);
    switch (slot >> 2) {
    case 0: return Ta * Tc * (p.rho * q.rho * ww);
    case 1: return Da * Dc * ww;
    case 2: return Da * Tc * ww;
    case 3: return Ta * Dc * ww;
    default: return Ta * Tc * ww;
    }
}

// Shared-memory layout of the moment kernels (sizes from the host: nm modes, nsl slots).
//   acc[nm * nsl]   running moments of the CTA's element pair / work item
//   red[S * nm * 5] per-group partial sums of G_n and K^n_uv
//   fac[nsl]        the current point pair's factors
//   sum[nm * 5]     G_n, K^n_uv of the current point pair
template <bool MFIE>
__device__ __forceinline__ void bor_fold_pair(int nm, int S, double2 *red, double2 *sum, const double *fac,
                                              double2 *acc) {
    constexpr int NV = MFIE ? 5 : 1, nsl = MFIE ? BOR_ALL_SLOTS : BOR_SLOTS;
    const int t = threadIdx.x;
    // reduce the groups in a fixed order
    for (int i = t; i < nm * NV; i += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        for (int gq = 0; gq < S; ++gq) {
            const double2 r = red[gq * nm * NV + i];
            v.x += r.x;
            v.y += r.y;
        }
        sum[i] = v;
    }
    __syncthreads();
    for (int i = t; i < nm * nsl; i += blockDim.x) {
        const int n = i / nsl, slot = i - n * nsl;
        double2 v;
        if (slot < BOR_SLOTS) {
            v = sum[n * NV];
        } else {
            const int uv = (slot - BOR_SLOTS) >> 2;
            const double2 kv = sum[n * NV + 1 + uv];
            // odd brackets: K = -j sum F sin(n xi)
            v = (uv == 1 || uv == 2) ? make_double2(kv.y, -kv.x) : kv;
        }
        const double f = fac[slot];
        acc[i].x += f * v.x;
        acc[i].y += f * v.y;
    }
    __syncthreads();
}

// grid = (ne, ne), BOR_THREADS threads; pairs with cls != 0 return at once.  Thread
// (n = t % nm, grp = t / nm) sums mode n over the samples i = grp (mod S) of each point pair,
// with e^{j n xi_i} carried by rotation and re-anchored exactly every 32 of them; the groups'
// sums of each of the 9 point pairs are reduced in shared memory, and the 36 slot moments
// are formed once at the end.
// dynamic smem: samples [NV][BOR_FAR_CHUNK], red[S][nm][NV], sums[9][nm][NV], fac[9][nsl].
template <bool MFIE>
__global__ void __launch_bounds__(BOR_THREADS, 2)
k_bor_far(int ne, const double *__restrict__ nodes, const unsigned char *__restrict__ cls, double k, int mmax,
          int nxi_cap, double2 *__restrict__ mom, double2 *__restrict__ momk) {
    constexpr int NV = MFIE ? 5 : 1, nsl = MFIE ? BOR_ALL_SLOTS : BOR_SLOTS;
    constexpr int NPP = BOR_FAR_ORDER * BOR_FAR_ORDER;
    const int e = blockIdx.x, f = blockIdx.y;
    if (cls[(int64_t)e * ne + f] != 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nm = mmax + 2, S = BOR_THREADS / nm;
    double2 *chunk = reinterpret_cast<double2 *>(smem_raw);  // [NV][BOR_FAR_CHUNK]
    double2 *red = chunk + NV * BOR_FAR_CHUNK;                // [S][nm][NV]
    double2 *sums = red + S * nm * NV;                         // [NPP][nm][NV]
    double *fac = reinterpret_cast<double *>(sums + NPP * nm * NV);  // [NPP][nsl]
    const int t = threadIdx.x, n = t % nm, grp = t / nm;
    for (int pp = 0; pp < NPP; ++pp) {
        const int ip = pp / BOR_FAR_ORDER, iq = pp % BOR_FAR_ORDER;
        double xo, wo, xs, wsq;
        gl_node(BOR_FAR_ORDER, ip, xo, wo);
        gl_node(BOR_FAR_ORDER, iq, xs, wsq);
        const BorPt p = bor_point(nodes, e, 0.5 * (xo + 1.0), 0.5 * wo);
        const BorPt q = bor_point(nodes, f, 0.5 * (xs + 1.0), 0.5 * wsq);
        if (t < nsl) fac[pp * nsl + t] = bor_factor(p, q, t);
        const BorPair pr = bor_pair(k, p, q);
        const int N = min(bor_nxi(k, p.rho, q.rho, sqrt(pr.d2), mmax), nxi_cap);
        const double dxi = 2.0 * GRIM_PI / N;
        double2 sg = make_double2(0.0, 0.0), s1 = sg, s2 = sg, s3 = sg, s4 = sg;
        // rotation by n S samples (n < 128, N <= 8192: 32-bit phase indices)
        double rs, rc;
        sincospi(2.0 * (double)((n * S) % N) / N, &rs, &rc);
        for (int i0 = 0; i0 < N; i0 += BOR_FAR_CHUNK) {
            const int cnt = min(BOR_FAR_CHUNK, N - i0);
            __syncthreads();
            for (int j = t; j < cnt; j += blockDim.x) {
                const int i = i0 + j;
                double sh, ch;
                sincospi(i / (double)N, &sh, &ch);
                double2 g, F[4];
                bor_sample<MFIE>(pr, sh, 2.0 * sh * ch, dxi, g, F);
                chunk[j] = g;
                if constexpr (MFIE) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) chunk[(1 + u) * BOR_FAR_CHUNK + j] = F[u];
                }
            }
            __syncthreads();
            if (grp < S) {
                // samples i = grp (mod S); e^{j n xi_i} anchored exactly every 32 of them
                int j = (grp - i0 % S + S) % S;
                while (j < cnt) {
                    double zs, zc;
                    sincospi(2.0 * (double)((n * (i0 + j)) % N) / N, &zs, &zc);
                    double2 z = make_double2(zc, zs);
                    const int jend = min(cnt, j + 32 * S);
#pragma unroll(MFIE ? 2 : 4)
                    for (; j < jend; j += S) {
                        const double2 v = chunk[j];
                        sg.x += v.x * z.x;
                        sg.y += v.y * z.x;
                        if constexpr (MFIE) {
                            const double2 f0 = chunk[BOR_FAR_CHUNK + j], f1 = chunk[2 * BOR_FAR_CHUNK + j];
                            const double2 f2 = chunk[3 * BOR_FAR_CHUNK + j], f3 = chunk[4 * BOR_FAR_CHUNK + j];
                            s1.x += f0.x * z.x; s1.y += f0.y * z.x;
                            s2.x += f1.x * z.y; s2.y += f1.y * z.y;
                            s3.x += f2.x * z.y; s3.y += f2.y * z.y;
                            s4.x += f3.x * z.x; s4.y += f3.y * z.x;
                        }
                        z = make_double2(z.x * rc - z.y * rs, z.x * rs + z.y * rc);
                    }
                }
            }
        }
        if (grp < S) {
            double2 *r = red + (grp * nm + n) * NV;
            r[0] = sg;
            if constexpr (MFIE) {
                r[1] = s1;
                r[2] = s2;
                r[3] = s3;
                r[4] = s4;
            }
        }
        __syncthreads();
        for (int i = t; i < nm * NV; i += blockDim.x) {
            double2 v = make_double2(0.0, 0.0);
            for (int gq = 0; gq < S; ++gq) {
                const double2 r = red[gq * nm * NV + i];
                v.x += r.x;
                v.y += r.y;
            }
            sums[pp * nm * NV + i] = v;
        }
    }
    __syncthreads();
    const int64_t base = ((int64_t)e * ne + f) * nm;
    for (int i = t; i < nm * nsl; i += blockDim.x) {
        const int nn_ = i / nsl, slot = i - nn_ * nsl;
        const int v = slot < BOR_SLOTS ? 0 : 1 + ((slot - BOR_SLOTS) >> 2);
        double2 a = make_double2(0.0, 0.0);
        for (int pp = 0; pp < NPP; ++pp) {
            const double fc = fac[pp * nsl + slot];
            const double2 sv = sums[(pp * nm + nn_) * NV + v];
            a.x += fc * sv.x;
            a.y += fc * sv.y;
        }
        if (slot < BOR_SLOTS) {
            mom[(base + nn_) * BOR_SLOTS + slot] = a;
        } else {
            // odd brackets: K = -j (sine sum)
            if (v == 2 || v == 3) a = make_double2(a.y, -a.x);
            momk[(base + nn_) * BOR_KSLOTS + slot - BOR_SLOTS] = a;
        }
    }
}

// Near-pair xi rule on [0, pi] for delta = R0 / c, span = 4 pi / (nmax + k c + 1) (two
// periods of the fastest oscillation per panel):
// a sinh-mapped Gauss core on [0, a], a = min(4 delta, span, pi), then panels
// [a 2^g, a 2^(g+1)] while a 2^g < span, then panels of length span up to pi.
struct BorRule {
    double delta, span, a, vmax, top;
    int geo, uni;
};

__device__ __forceinline__ BorRule bor_rule(double delta, double span) {
    BorRule r;
    r.delta = delta;
    r.span = span;
    r.a = fmin(fmin(4.0 * delta, span), GRIM_PI);
    r.vmax = asinh(r.a / delta);
    r.geo = 0;
    double top = r.a;
    while (top < span && top < GRIM_PI && r.geo < 2048) {
        top *= 2.0;
        ++r.geo;
    }
    r.top = top;
    int uni = top < GRIM_PI ? (int)ceil((GRIM_PI - top) / span) : 0;
    if (uni > 0 && top + (uni - 1) * span >= GRIM_PI) --uni;
    r.uni = uni;
    return r;
}

__device__ __forceinline__ int bor_rule_count(const BorRule &r) { return BOR_XI_CORE + BOR_XI_PANEL * (r.geo + r.uni); }

// Node j of the rule: xi and weight (times 2 for the half range).
__device__ __forceinline__ void bor_rule_node(const BorRule &r, int j, double &xi, double &w) {
    double x, wg;
    if (j < BOR_XI_CORE) {
        gl_node(BOR_XI_CORE, j, x, wg);
        const double v = 0.5 * (x + 1.0) * r.vmax;
        xi = r.delta * sinh(v);
        w = r.delta * cosh(v) * (0.5 * wg) * r.vmax;
    } else {
        const int P = (j - BOR_XI_CORE) / BOR_XI_PANEL, q = (j - BOR_XI_CORE) % BOR_XI_PANEL;
        double lo, hi;
        if (P < r.geo) {
            lo = ldexp(r.a, P);
            hi = fmin(ldexp(r.a, P + 1), GRIM_PI);
        } else {
            lo = fmin(r.top + (P - r.geo) * r.span, GRIM_PI);
            hi = fmin(r.top + (P + 1 - r.geo) * r.span, GRIM_PI);
        }
        gl_node(BOR_XI_PANEL, q, x, wg);
        xi = lo + (hi - lo) * (0.5 * (x + 1.0));
        w = (hi - lo) * (0.5 * wg);
    }
    w *= 2.0;
}

struct BorItem {
    int e, f, r0, r1;  // element pair and its point-pair range in the rule table
};

#define BOR_NEAR_EVAL 256  // near-rule samples evaluated per pass (one per thread)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// grid = number of near work items, BOR_THREADS threads.  rule[3 i .. 3 i + 2] = (s, s', w).
// Writes the item's moments to part[item][n][slot] (nm x nsl complex).  Per point pair the
// rule's samples are evaluated BOR_NEAR_EVAL at a time (one per thread, with e^{j xi} and
// e^{j Q xi}, Q = ceil(nm / 4)); rows e^{j n xi} of chr samples at a time are then built by
// rotation (four threads per sample, one quarter of the orders each) and summed by the
// (mode, group) threads.
// dynamic smem: smp[NV][BOR_NEAR_EVAL], z1[BOR_NEAR_EVAL], zq[BOR_NEAR_EVAL],
// rot[chr][P] (P = nm rounded up to odd: conflict-free row writes; the groups' partial
// sums red[S][nm][NV] reuse it once a point pair's rows are consumed), then sum, acc, fac.
template <bool MFIE>
__global__ void __launch_bounds__(BOR_THREADS, 2)
k_bor_near(const BorItem *__restrict__ items, const double *__restrict__ nodes, const double *__restrict__ rule,
           double k, int mmax, int chr, double2 *__restrict__ part) {
    constexpr int NV = MFIE ? 5 : 1, nsl = MFIE ? BOR_ALL_SLOTS : BOR_SLOTS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nm = mmax + 2, S = BOR_THREADS / nm, P = nm | 1, Q = (nm + 3) / 4;
    double2 *smp = reinterpret_cast<double2 *>(smem_raw);  // [NV][BOR_NEAR_EVAL]
    double2 *sz1 = smp + NV * BOR_NEAR_EVAL;
    double2 *szq = sz1 + BOR_NEAR_EVAL;
    double2 *rot = szq + BOR_NEAR_EVAL;                     // [chr][P]
    double2 *red = rot;                                     // [S][nm][NV], after the rows
    double2 *sum = rot + max(chr * P, S * nm * NV);
    double2 *acc = sum + nm * NV;
    double *fac = reinterpret_cast<double *>(acc + nm * nsl);
    const BorItem it = items[blockIdx.x];
    const int t = threadIdx.x, n = t % nm, grp = t / nm;
    for (int i = t; i < nm * nsl; i += blockDim.x) acc[i] = make_double2(0.0, 0.0);
    for (int ipp = it.r0; ipp < it.r1; ++ipp) {
        const BorPt p = bor_point(nodes, it.e, rule[3 * ipp], rule[3 * ipp + 2]);
        const BorPt q = bor_point(nodes, it.f, rule[3 * ipp + 1], 1.0);
        const BorPair pr = bor_pair(k, p, q);
        const double c = sqrt(p.rho * q.rho);
        const BorRule rl = bor_rule(sqrt(pr.d2) / c, 4.0 * GRIM_PI / ((mmax + 1) + k * c + 1.0));
        const int na = bor_rule_count(rl);
        if (t < nsl) fac[t] = bor_factor(p, q, t);
        double2 sg = make_double2(0.0, 0.0), s1 = sg, s2 = sg, s3 = sg, s4 = sg;
        for (int j0 = 0; j0 < na; j0 += BOR_NEAR_EVAL) {
            const int cnt = min(BOR_NEAR_EVAL, na - j0);
            __syncthreads();
            for (int j = t; j < cnt; j += blockDim.x) {
                double xi, w;
                bor_rule_node(rl, j0 + j, xi, w);
                double sh, ch;
                sincos(0.5 * xi, &sh, &ch);
                double2 g, F[4];
                bor_sample<MFIE>(pr, sh, 2.0 * sh * ch, w, g, F);
                smp[j] = g;
                if constexpr (MFIE) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) smp[(1 + u) * BOR_NEAR_EVAL + j] = F[u];
                }
                // e^{j xi} and e^{j Q xi} (binary powers)
                const double2 z1 = make_double2(1.0 - 2.0 * sh * sh, 2.0 * sh * ch);
                double2 zq = make_double2(1.0, 0.0), b = z1;
                for (int e2 = Q; e2 > 0; e2 >>= 1) {
                    if (e2 & 1) zq = cmul(zq, b);
                    b = cmul(b, b);
                }
                sz1[j] = z1;
                szq[j] = zq;
            }
            for (int s0 = 0; s0 < cnt; s0 += chr) {
                const int sc = min(chr, cnt - s0);
                __syncthreads();
                for (int task = t; task < 4 * sc; task += blockDim.x) {
                    const int jj = task % sc, quarter = task / sc;
                    const int n0 = quarter * Q, n1 = min(nm, n0 + Q);
                    if (n0 >= n1) continue;
                    const double2 z1 = sz1[s0 + jj], zq = szq[s0 + jj];
                    double2 z = make_double2(1.0, 0.0);
                    for (int r = 0; r < quarter; ++r) z = cmul(z, zq);
                    double2 *row = rot + jj * P;
                    for (int nn_ = n0; nn_ < n1; ++nn_) {
                        row[nn_] = z;
                        z = cmul(z, z1);
                    }
                }
                __syncthreads();
                if (grp < S) {
#pragma unroll 4
                    for (int jj = grp; jj < sc; jj += S) {
                        const double2 z = rot[jj * P + n];
                        const int j = s0 + jj;
                        const double2 v = smp[j];
                        sg.x += v.x * z.x;
                        sg.y += v.y * z.x;
                        if constexpr (MFIE) {
                            const double2 f0 = smp[BOR_NEAR_EVAL + j], f1 = smp[2 * BOR_NEAR_EVAL + j];
                            const double2 f2 = smp[3 * BOR_NEAR_EVAL + j], f3 = smp[4 * BOR_NEAR_EVAL + j];
                            s1.x += f0.x * z.x; s1.y += f0.y * z.x;
                            s2.x += f1.x * z.y; s2.y += f1.y * z.y;
                            s3.x += f2.x * z.y; s3.y += f2.y * z.y;
                            s4.x += f3.x * z.x; s4.y += f3.y * z.x;
                        }
                    }
                }
            }
        }
        __syncthreads();  // every thread is done with the rows that red overwrites
        if (grp < S) {
            double2 *r = red + (grp * nm + n) * NV;
            r[0] = sg;
            if constexpr (MFIE) {
                r[1] = s1;
                r[2] = s2;
                r[3] = s3;
                r[4] = s4;
            }
        }
        __syncthreads();
        bor_fold_pair<MFIE>(nm, S, red, sum, fac, acc);
    }
    double2 *out = part + (int64_t)blockIdx.x * nm * nsl;
    for (int i = t; i < nm * nsl; i += blockDim.x) out[i] = acc[i];
}

// grid = number of near element pairs; pairs[i] = (e, f, first item, end item).
template <bool MFIE>
__global__ void k_bor_near_reduce(int ne, int mmax, const int4 *__restrict__ pairs, const double2 *__restrict__ part,
                                  double2 *__restrict__ mom, double2 *__restrict__ momk) {
    constexpr int nsl = MFIE ? BOR_ALL_SLOTS : BOR_SLOTS;
    const int nm = mmax + 2;
    const int4 pq = pairs[blockIdx.x];
    const int64_t base = ((int64_t)pq.x * ne + pq.y) * nm;
    for (int i = threadIdx.x; i < nm * nsl; i += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        for (int it = pq.z; it < pq.w; ++it) {
            const double2 r = part[(int64_t)it * nm * nsl + i];
            v.x += r.x;
            v.y += r.y;
        }
        const int nn_ = i / nsl, slot = i - nn_ * nsl;
        if (slot < BOR_SLOTS) mom[(base + nn_) * BOR_SLOTS + slot] = v;
        else momk[(base + nn_) * BOR_KSLOTS + slot - BOR_SLOTS] = v;
    }
}

// grid = ceil(nred / 16) x ceil(nred / 16), block 16 x 16.  red_full[2*nred] lists, for
// every reduced function, up to two full components (t: node, phi: nn + node; -1 unused)
// and red_w[2*nred] their complex weights (1, or j m sign(t_rho) for a pole phi folded into
// the pole t function).  Each entry is sum over the components of conj(w_row) Z_full w_col
// with Z_full = alpha C EFIE + beta ((1/2) M - K) (beta = (1 - alpha) eta0; momk == nullptr
// for the EFIE alone, alpha = 1).
__global__ void k_bor_assemble(int ne, int mmax, int m, double k, const double2 *__restrict__ mom,
                               const double2 *__restrict__ momk, double alpha, int nred,
                               const int *__restrict__ red_full, const double2 *__restrict__ red_w,
                               const double *__restrict__ nodes, double2 *__restrict__ Z, int64_t ldz) {
    const int r = blockIdx.x * 16 + threadIdx.x;  // row (test)
    const int c = blockIdx.y * 16 + threadIdx.y;  // column (source)
    if (r >= nred || c >= nred) return;
    const int nn = ne + 1;
    const int nm = mmax + 2;
    const int am = abs(m), am1 = abs(m - 1), ap1 = abs(m + 1);
    const double km2 = 1.0 / (k * k);
    const double C = k * 376.730313668 * 2.0 * GRIM_PI;  // C = j k eta 2 pi (times j below)
    const double beta = momk ? (1.0 - alpha) * 376.730313668 : 0.0;
    double2 total = make_double2(0.0, 0.0);
    for (int ri = 0; ri < 2; ++ri) {
        const int fr = red_full[2 * r + ri];
        if (fr < 0) continue;
        const double2 wr = red_w[2 * r + ri];
        const int ni = fr % nn, ci = fr / nn;  // node, component (0 t, 1 phi)
        for (int cj = 0; cj < 2; ++cj) {
            const int fc = red_full[2 * c + cj];
            if (fc < 0) continue;
            const double2 wc = red_w[2 * c + cj];
            const int nj = fc % nn, cc = fc / nn;
            double2 z = make_double2(0.0, 0.0), zk = z;
            double mass = 0.0;
            // element pairs (e, f) with e in {ni-1, ni}, f in {nj-1, nj}
            for (int de = 0; de < 2; ++de) {
                const int e = ni - 1 + de;
                if (e < 0 || e >= ne) continue;
                const int a = 1 - de;  // node ni is node index a of element e (e = ni-1 -> a = 1)
                const double dre = nodes[2 * e + 2] - nodes[2 * e], dze = nodes[2 * e + 3] - nodes[2 * e + 1];
                const double Le = hypot(dre, dze), tre = dre / Le, tze = dze / Le;
                for (int df = 0; df < 2; ++df) {
                    const int f = nj - 1 + df;
                    if (f < 0 || f >= ne) continue;
                    const int b = 1 - df;
                    const double drf = nodes[2 * f + 2] - nodes[2 * f], dzf = nodes[2 * f + 3] - nodes[2 * f + 1];
                    const double Lf = hypot(drf, dzf), trf = drf / Lf, tzf = dzf / Lf;
                    const int s = 2 * a + b;
                    const double2 *base = mom + ((int64_t)e * ne + f) * nm * BOR_SLOTS;
                    const double2 A0 = base[am * BOR_SLOTS + s];
                    const double2 Am1 = base[am1 * BOR_SLOTS + s];
                    const double2 Ap1 = base[ap1 * BOR_SLOTS + s];
                    const double2 Ac = make_double2(0.5 * (Am1.x + Ap1.x), 0.5 * (Am1.y + Ap1.y));
                    const double2 As = make_double2(0.5 * (Am1.x - Ap1.x), 0.5 * (Am1.y - Ap1.y));
                    const double2 DD = base[am * BOR_SLOTS + 4 + s];
                    const double2 DT = base[am * BOR_SLOTS + 8 + s];
                    const double2 TD = base[am * BOR_SLOTS + 12 + s];
                    const double2 TT = base[am * BOR_SLOTS + 16 + s];
                    double2 v;
                    if (ci == 0 && cc == 0) {
                        v.x = tre * trf * Ac.x + tze * tzf * A0.x - km2 * DD.x;
                        v.y = tre * trf * Ac.y + tze * tzf * A0.y - km2 * DD.y;
                    } else if (ci == 0 && cc == 1) {  // -j tre As - (j m / k^2) DT
                        v.x = tre * As.y + m * km2 * DT.y;
                        v.y = -tre * As.x - m * km2 * DT.x;
                    } else if (ci == 1 && cc == 0) {  // +j trf As + (j m / k^2) TD
                        v.x = -trf * As.y - m * km2 * TD.y;
                        v.y = trf * As.x + m * km2 * TD.x;
                    } else {                          // Ac - (m^2 / k^2) TT
                        v.x = Ac.x - (double)m * m * km2 * TT.x;
                        v.y = Ac.y - (double)m * m * km2 * TT.y;
                    }
                    z.x += v.x;
                    z.y += v.y;
                    if (momk) {
                        // K of quadrant uv (tt, tf, ft, ff); odd quadrants change sign with m
                        const int uv = 2 * ci + cc;
                        const double sg = (m < 0 && (uv == 1 || uv == 2)) ? -1.0 : 1.0;
                        const double2 kv =
                            momk[(((int64_t)e * ne + f) * nm + am) * BOR_KSLOTS + 4 * uv + s];
                        zk.x += sg * kv.x;
                        zk.y += sg * kv.y;
                        if (e == f && ci == cc) {
                            // mass 2 pi int rho T_a T_b dt on element e (3-point Gauss)
                            for (int ip = 0; ip < BOR_FAR_ORDER; ++ip) {
                                double xg, wg;
                                gl_node(BOR_FAR_ORDER, ip, xg, wg);
                                const double sq = 0.5 * (xg + 1.0);
                                const double rho = nodes[2 * e] + sq * dre;
                                const double Ta = a ? sq : 1.0 - sq, Tb = b ? sq : 1.0 - sq;
                                mass += 2.0 * GRIM_PI * (0.5 * wg * Le) * rho * Ta * Tb;
                            }
                        }
                    }
                }
            }
            // Z_full = alpha C j z + beta ((1/2) mass - 2 pi zk)
            double2 v = make_double2(-alpha * C * z.y, alpha * C * z.x);
            if (momk) {
                v.x += beta * (0.5 * mass - 2.0 * GRIM_PI * zk.x);
                v.y += beta * (-2.0 * GRIM_PI * zk.y);
            }
            // conj(wr) * v * wc
            const double2 t1 = make_double2(wr.x * v.x + wr.y * v.y, wr.x * v.y - wr.y * v.x);
            total.x += t1.x * wc.x - t1.y * wc.y;
            total.y += t1.x * wc.y + t1.y * wc.x;
        }
    }
    Z[(int64_t)c * ldz + r] = total;
}

// J_m(x) for any integer m (J_{-m} = (-1)^m J_m), through CUDA's jn.
__device__ __forceinline__ double jn_signed(int m, double x) {
    if (x == 0.0) return m == 0 ? 1.0 : 0.0;  // on-axis aspects: J_n(0) = delta_n0
    if (m >= 0) return jn(m, x);
    const double v = jn(-m, x);
    return ((-m) & 1) ? -v : v;
}

// Per (aspect, Gauss point): J_m, J_{m-1}, J_{m+1} at k rho sin(theta) and the axial phase
// e^{j k z cos(theta)} -- evaluated once and shared by every row that the point touches.
// tab[((it * ne + e) * BOR_FAR_ORDER + ip) * 5 + {0..4}] = (J_m, J_{m-1}, J_{m+1}, cos, sin).
__global__ void k_bor_bessel(int ne, const double *__restrict__ nodes, double k, int m, int nth,
                             const double *__restrict__ th_deg, double *__restrict__ tab) {
    const int pidx = blockIdx.x * blockDim.x + threadIdx.x;
    const int it = blockIdx.y;
    if (pidx >= ne * BOR_FAR_ORDER || it >= nth) return;
    const int e = pidx / BOR_FAR_ORDER, ip = pidx % BOR_FAR_ORDER;
    double st, ct;
    sincospi(th_deg[it] / 180.0, &st, &ct);
    double xg, wg;
    gl_node(BOR_FAR_ORDER, ip, xg, wg);
    const double s = 0.5 * (xg + 1.0);
    const double r0 = nodes[2 * e], z0 = nodes[2 * e + 1];
    const double rho = r0 + s * (nodes[2 * e + 2] - r0), z = z0 + s * (nodes[2 * e + 3] - z0);
    const double x = k * rho * st;
    double *o = tab + ((int64_t)it * ne * BOR_FAR_ORDER + pidx) * 5;
    o[0] = jn_signed(m, x);
    o[1] = jn_signed(m - 1, x);
    o[2] = jn_signed(m + 1, x);
    double sp, cp;
    sincos(k * z * ct, &sp, &cp);
    o[3] = cp;
    o[4] = sp;
}

// Reduced excitation (far = 0) or far-field weights (far = 1) for mode m, from the
// k_bor_bessel table of the same (m, aspects).
// Columns: [VV theta_0..n-1, HH theta_0..n-1].  One thread per (reduced row, column).
__global__ void k_bor_excitation(int ne, const double *__restrict__ nodes, int m, int nth,
                                 const double *__restrict__ th_deg, const double *__restrict__ tab, int far,
                                 double alpha, int nred, const int *__restrict__ red_full,
                                 const double2 *__restrict__ red_w, double2 *__restrict__ V, int64_t ldv) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int col = blockIdx.y;
    if (r >= nred || col >= 2 * nth) return;
    const int nn = ne + 1;
    const int it = col % nth;
    const bool hh = col >= nth;
    double st, ct;
    sincospi(th_deg[it] / 180.0, &st, &ct);
    double2 total = make_double2(0.0, 0.0);
    for (int ri = 0; ri < 2; ++ri) {
        const int fr = red_full[2 * r + ri];
        if (fr < 0) continue;
        const double2 w = red_w[2 * r + ri];
        const int node = fr % nn, comp = fr / nn;
        double2 sum = make_double2(0.0, 0.0);
        for (int de = 0; de < 2; ++de) {
            const int e = node - 1 + de;
            if (e < 0 || e >= ne) continue;
            const int a = 1 - de;
            const double r0 = nodes[2 * e], dr = nodes[2 * e + 2] - r0, dz = nodes[2 * e + 3] - nodes[2 * e + 1];
            const double L = hypot(dr, dz), tr = dr / L, tz = dz / L;
            for (int ip = 0; ip < BOR_FAR_ORDER; ++ip) {
                double xg, wg;
                gl_node(BOR_FAR_ORDER, ip, xg, wg);
                const double s = 0.5 * (xg + 1.0);
                const double rho = r0 + s * dr, w = 0.5 * wg * L;
                const double T = a == 0 ? 1.0 - s : s;
                const double *tb = tab + (((int64_t)it * ne + e) * BOR_FAR_ORDER + ip) * 5;
                const double jm = tb[0], jm1 = tb[1], jp1 = tb[2];
                // j^m, j^(m-1), j^(m+1) as unit complex numbers
                const int q0 = ((m % 4) + 4) % 4, qm = (((m - 1) % 4) + 4) % 4, qp = (((m + 1) % 4) + 4) % 4;
                const double2 u0 = make_double2(q0 == 0 ? 1 : (q0 == 2 ? -1 : 0), q0 == 1 ? 1 : (q0 == 3 ? -1 : 0));
                const double2 um = make_double2(qm == 0 ? 1 : (qm == 2 ? -1 : 0), qm == 1 ? 1 : (qm == 3 ? -1 : 0));
                const double2 up = make_double2(qp == 0 ? 1 : (qp == 2 ? -1 : 0), qp == 1 ? 1 : (qp == 3 ? -1 : 0));
                const double2 I0 = make_double2(2 * GRIM_PI * u0.x * jm, 2 * GRIM_PI * u0.y * jm);
                const double2 Ic = make_double2(GRIM_PI * (up.x * jp1 + um.x * jm1), GRIM_PI * (up.y * jp1 + um.y * jm1));
                // Is = -j pi (j^(m-1) J_{m-1} - j^(m+1) J_{m+1})
                const double2 dd = make_double2(um.x * jm1 - up.x * jp1, um.y * jm1 - up.y * jp1);
                double2 Is = make_double2(GRIM_PI * dd.y, -GRIM_PI * dd.x);
                if (far) Is = make_double2(-Is.x, -Is.y);
                double2 ang;
                if (!hh) {
                    if (comp == 0) ang = make_double2(tr * ct * Ic.x - tz * st * I0.x, tr * ct * Ic.y - tz * st * I0.y);
                    else ang = make_double2(-ct * Is.x, -ct * Is.y);
                } else {
                    if (comp == 0) ang = make_double2(tr * Is.x, tr * Is.y);
                    else ang = Ic;
                }
                if (!far && alpha != 1.0) {
                    // eta0 <W, n x H_inc> (reference rhs_mfie_mode), weighted 1 - alpha
                    double2 hm;
                    if (!hh) {
                        if (comp == 0) hm = Ic;
                        else hm = make_double2(-tr * Is.x, -tr * Is.y);
                    } else {
                        if (comp == 0) hm = make_double2(ct * Is.x, ct * Is.y);
                        else hm = make_double2(tr * ct * Ic.x - tz * st * I0.x, tr * ct * Ic.y - tz * st * I0.y);
                    }
                    ang = make_double2(alpha * ang.x + (1.0 - alpha) * hm.x, alpha * ang.y + (1.0 - alpha) * hm.y);
                }
                const double cp = tb[3], sp = tb[4];
                const double f = rho * w * T;
                const double2 ph = make_double2(cp * f, sp * f);
                sum.x += ph.x * ang.x - ph.y * ang.y;
                sum.y += ph.x * ang.y + ph.y * ang.x;
            }
        }
        // rhs: conj(w) * sum (Q^H V);  far weights: w * sum (Q^T W)
        if (far) {
            total.x += w.x * sum.x - w.y * sum.y;
            total.y += w.x * sum.y + w.y * sum.x;
        } else {
            total.x += w.x * sum.x + w.y * sum.y;
            total.y += w.x * sum.y - w.y * sum.x;
        }
    }
    V[(int64_t)col * ldv + r] = total;
}

// amp[col] += sum_r W[r, col] * X[r, col]  (one CTA per column, fixed-order reduction)
__global__ void k_bor_farfield_accumulate(int nred, int ncol, const double2 *__restrict__ W, int64_t ldw,
                                          const double2 *__restrict__ X, int64_t ldx, double2 *__restrict__ amp) {
    const int col = blockIdx.x;
    double re = 0.0, im = 0.0;
    for (int r = threadIdx.x; r < nred; r += blockDim.x) {
        const double2 w = W[(int64_t)col * ldw + r], x = X[(int64_t)col * ldx + r];
        re += w.x * x.x - w.y * x.y;
        im += w.x * x.y + w.y * x.x;
    }
    for (int off = 16; off > 0; off >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, off);
        im += __shfl_down_sync(0xffffffffu, im, off);
    }
    __shared__ double sr[32], si[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sr[warp] = re; si[warp] = im; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        re = lane < nw ? sr[lane] : 0.0;
        im = lane < nw ? si[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) {
            re += __shfl_down_sync(0xffffffffu, re, off);
            im += __shfl_down_sync(0xffffffffu, im, off);
        }
        if (lane == 0) {
            amp[col].x += re;
            amp[col].y += im;
        }
    }
}

// ---- mirror-symmetric bodies: even / odd halves of a mode system (reference
// bor/factor.py:37-116 MirrorSplit).  A body symmetric about a plane normal to the axis
// maps reduced unknown u to target[u] with sign[u] (J_t changes sign, J_phi does not).
// Pairs (p1 < p2 = target[p1], s = sign[p2]) and fixed unknowns (fe: sign +1, fo: sign -1)
// give, with r = 1/sqrt(2), the even half over (r (u_p1 + s u_p2), u_fe) and the odd half
// over (r (u_p1 - s u_p2), u_fo); when A = R A R they decouple exactly:
//   H[:k,:k] = (a[p1,p1] + s a[p2,p2] s +- (a[p1,p2] s + s a[p2,p1])) / 2
//   H[:k,k:] = (a[p1,f] +- s a[p2,f]) r,  H[k:,:k] = (a[f,p1] +- a[f,p2] s) r,  H[k:,k:] = a[f,f].
struct BorMirror {
    int k, nfe, nfo;
    const int *p1, *p2, *fe, *fo;
    const double *s;
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double f) { return make_double2(a.x * f, a.y * f); }

// grid over the (ke x ke) even and (ko x ko) odd halves; He, Ho column-major (ld ke, ko).
__global__ void k_bor_mirror_halves(BorMirror mr, const double2 *__restrict__ Z, int64_t ldz, double2 *__restrict__ He,
                                    double2 *__restrict__ Ho) {
    const int i = blockIdx.x * 16 + threadIdx.x, j = blockIdx.y * 16 + threadIdx.y;
    const int k = mr.k, ke = k + mr.nfe, ko = k + mr.nfo;
    const double r = 0.7071067811865475244;
    auto a = [&](int row, int col) { return Z[(int64_t)col * ldz + row]; };
    for (int parity = 0; parity < 2; ++parity) {
        const int m = parity ? ko : ke;
        if (i >= m || j >= m) continue;
        const double sg = parity ? -1.0 : 1.0;
        const int *fx = parity ? mr.fo : mr.fe;
        double2 v;
        if (i < k && j < k) {
            const int a1 = mr.p1[i], a2 = mr.p2[i], b1 = mr.p1[j], b2 = mr.p2[j];
            const double si = mr.s[i], sj = mr.s[j];
            const double2 common = cadd(a(a1, b1), cscale(a(a2, b2), si * sj));
            const double2 cross = cadd(cscale(a(a1, b2), sj), cscale(a(a2, b1), si));
            v = cscale(cadd(common, cscale(cross, sg)), 0.5);
        } else if (i < k) {
            const int f = fx[j - k];
            v = cscale(cadd(a(mr.p1[i], f), cscale(a(mr.p2[i], f), sg * mr.s[i])), r);
        } else if (j < k) {
            const int f = fx[i - k];
            v = cscale(cadd(a(f, mr.p1[j]), cscale(a(f, mr.p2[j]), sg * mr.s[j])), r);
        } else {
            v = a(fx[i - k], fx[j - k]);
        }
        (parity ? Ho : He)[(int64_t)j * m + i] = v;
    }
}

// max over entries of |a - (R A R)| and of |a| (two non-negative doubles, as ordered bits).
__global__ void k_bor_mirror_asym(int n, const double2 *__restrict__ Z, int64_t ldz, const int *__restrict__ target,
                                  const double *__restrict__ sign, unsigned long long *__restrict__ out) {
    const int i = blockIdx.x * 16 + threadIdx.x, j = blockIdx.y * 16 + threadIdx.y;
    double d = 0.0, m = 0.0;
    if (i < n && j < n) {
        const double2 a = Z[(int64_t)j * ldz + i];
        const double2 b = Z[(int64_t)target[j] * ldz + target[i]];
        const double f = sign[i] * sign[j];
        d = hypot(a.x - f * b.x, a.y - f * b.y);
        m = hypot(a.x, a.y);
    }
    for (int off = 16; off > 0; off >>= 1) {
        d = fmax(d, __shfl_down_sync(0xffffffffu, d, off));
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    }
    if ((threadIdx.x + 16 * threadIdx.y) % 32 == 0) {
        atomicMax(out, (unsigned long long)__double_as_longlong(d));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong(m));
    }
}

// Right-hand sides (n x nrhs, ld ldb) into the even (ke x nrhs) and odd (ko x nrhs) parts.
__global__ void k_bor_mirror_split(BorMirror mr, int nrhs, const double2 *__restrict__ B, int64_t ldb,
                                   double2 *__restrict__ Be, double2 *__restrict__ Bo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    const int k = mr.k, ke = k + mr.nfe, ko = k + mr.nfo;
    if (c >= nrhs) return;
    const double r = 0.7071067811865475244;
    const double2 *b = B + (int64_t)c * ldb;
    if (i < ke) {
        Be[(int64_t)c * ke + i] = i < k ? cscale(cadd(b[mr.p1[i]], cscale(b[mr.p2[i]], mr.s[i])), r) : b[mr.fe[i - k]];
    }
    if (i < ko) {
        Bo[(int64_t)c * ko + i] = i < k ? cscale(cadd(b[mr.p1[i]], cscale(b[mr.p2[i]], -mr.s[i])), r) : b[mr.fo[i - k]];
    }
}

// Solutions of the halves back to the n unknowns.
__global__ void k_bor_mirror_join(BorMirror mr, int nrhs, const double2 *__restrict__ Ye,
                                  const double2 *__restrict__ Yo, double2 *__restrict__ X, int64_t ldx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    const int k = mr.k, ke = k + mr.nfe, ko = k + mr.nfo;
    if (c >= nrhs) return;
    const double r = 0.7071067811865475244;
    double2 *x = X + (int64_t)c * ldx;
    const double2 *ye = Ye + (int64_t)c * ke, *yo = Yo + (int64_t)c * ko;
    if (i < k) {
        const double2 e = ye[i], o = yo[i];
        x[mr.p1[i]] = cscale(cadd(e, o), r);
        x[mr.p2[i]] = cscale(cadd(e, cscale(o, -1.0)), r * mr.s[i]);
    } else if (i < ke && i - k < mr.nfe) {
        x[mr.fe[i - k]] = ye[i];
    }
    if (i >= k && i < ko) x[mr.fo[i - k]] = yo[i];
}
