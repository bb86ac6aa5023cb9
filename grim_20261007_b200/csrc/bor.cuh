// Body-of-revolution PEC EFIE, per azimuthal mode.
//
// Stage 1  k_bor_moments: one CTA per element pair (e, f).  For every point pair it
//   evaluates the modal Green's function G_n = int_0^{2pi} e^{-jkR}/(4 pi R) cos(n xi) dxi
//   for n = 0..mmax+1 (uniform trapezoid with a per-pair sample count for far pairs,
//   sinh-substituted Gauss rule for same/adjacent elements) and accumulates the 20
//   mode-independent element moments per n:
//     A_ac  = sum T_a T_c rho rho' w w' G_n      DD_ac = sum D_a D_c w w' G_n
//     DT_ac = sum D_a T_c w w' G_n               TD_ac = sum T_a D_c w w' G_n
//     TT_ac = sum T_a T_c w w' G_n               (a, c in {0, 1}: the element's two tents)
//   Layout: mom[((e * ne + f) * (mmax + 2) + n) * 20 + slot], complex128.
// Stage 2  k_bor_assemble: the reduced mode-m matrix from the moments of the <= 4
//   element pairs touching each node pair, with the pole treatment (inactive pole phi
//   components, |m| = 1 pole t component tied to phi by j m sign(t_rho)).
// Stage 3  k_bor_excitation: reduced right-hand sides (VV, HH per aspect) or far-field
//   weights, with the phi integrals in closed form through J_m (CUDA's jn).
// Reference: bor/solver.py:1769-1827 (assemble_mode), :2369-2440 (pole reduction),
// :2558-2608 (rhs_vv_hh_batch / farfield_vv_hh_batch), bor/kernels.py:632 (modal kernels).
#pragma once
#include "common.cuh"

#define BOR_FAR_ORDER 3
#define BOR_NEAR_ORDER 8
#define BOR_NEAR_XI 32
#define BOR_MAX_MODES 128
#define BOR_MAX_NXI 8192
#define BOR_SLOTS 20

struct BorPt {
    double rho, z, w, T0, T1, D0, D1;
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
    return p;
}

__device__ __forceinline__ int bor_nxi(double k, double rp, double rq, double r0, int mmax) {
    const double c = sqrt(rp * rq);
    const double v = 1.5 * (2.0 * k * c + mmax + 2) + 30.0 * c / fmax(r0, 1e-300) + 16.0;
    int n = 32 * (int)ceil(v / 32.0);
    return n > BOR_MAX_NXI ? BOR_MAX_NXI : n;
}

// Gauss-Legendre nodes/weights (orders 1..32) from the 2-D fill's constant tables.
__device__ __forceinline__ void gl_node(int q, int i, double &x, double &w) {
    x = c_gl_x[q * (q - 1) / 2 + i];
    w = c_gl_w[q * (q - 1) / 2 + i];
}

// Source rule for a near pair: point i of the cubically graded rule(s) on [0,1];
// self pairs split at s_obs (16 points), adjacent pairs cluster at the shared node.
__device__ __forceinline__ void near_src(int e, int f, double s_obs, int i, double &s, double &ws) {
    double x, w;
    if (e == f) {
        const int half = i / BOR_NEAR_ORDER, ii = i % BOR_NEAR_ORDER;
        gl_node(BOR_NEAR_ORDER, ii, x, w);
        const double u = 0.5 * (x + 1.0), wu = 0.5 * w;
        if (half == 0) {  // [0, s_obs] toward s_obs
            s = s_obs - s_obs * u * u * u;
            ws = s_obs * 3.0 * u * u * wu;
        } else {          // [s_obs, 1] toward s_obs
            s = s_obs + (1.0 - s_obs) * u * u * u;
            ws = (1.0 - s_obs) * 3.0 * u * u * wu;
        }
    } else {
        gl_node(BOR_NEAR_ORDER, i, x, w);
        const double u = 0.5 * (x + 1.0), wu = 0.5 * w;
        if (f == e + 1) {  // toward 0
            s = u * u * u;
        } else {           // toward 1
            s = 1.0 - u * u * u;
        }
        ws = 3.0 * u * u * wu;
    }
}

// One point pair: compute G_n (n = 0..nm-1) into sG and accumulate the 20 moments.
// All threads of the CTA participate; thread n < nm owns mode n's accumulators.
__device__ __forceinline__ void bor_pair_accumulate(double k, const BorPt &p, const BorPt &q, bool near, int mmax,
                                                    int nxi_cap, double2 *sg, double *scos, double2 *sG,
                                                    double2 (&acc)[BOR_SLOTS]) {
    const int t = threadIdx.x, nt = blockDim.x;
    const int nm = mmax + 2;
    const double r0 = sqrt((p.rho - q.rho) * (p.rho - q.rho) + (p.z - q.z) * (p.z - q.z));
    const double rr4 = 4.0 * p.rho * q.rho;
    double2 gsum = make_double2(0.0, 0.0);
    if (!near) {
        // nxi_cap = the shared-memory capacity the host sized (>= every far pair's count)
        const int N = min(bor_nxi(k, p.rho, q.rho, r0, mmax), nxi_cap);
        const double dxi = 2.0 * GRIM_PI / N;
        for (int i = t; i < N; i += nt) {
            double sx, cx;
            sincospi(2.0 * i / (double)N, &sx, &cx);
            scos[i] = cx;
            const double s2 = sin(0.5 * i * dxi);
            const double R = sqrt(r0 * r0 + rr4 * s2 * s2);
            double sk, ck;
            sincos(k * R, &sk, &ck);
            const double f = dxi / (4.0 * GRIM_PI * R);
            sg[i] = make_double2(ck * f, -sk * f);
        }
        __syncthreads();
        if (t < nm) {
            int idx = 0;
            for (int i = 0; i < N; ++i) {
                const double c = scos[idx];
                gsum.x += sg[i].x * c;
                gsum.y += sg[i].y * c;
                idx += t;
                if (idx >= N) idx -= N;
            }
            sG[t] = gsum;
        }
        __syncthreads();
    } else {
        const double c = sqrt(p.rho * q.rho);
        const double umax = asinh(c * GRIM_PI / fmax(r0, 1e-300));
        const double sc = fmax(r0, 1e-300) / c;
        for (int i = t; i < BOR_NEAR_XI; i += nt) {
            double x, w;
            gl_node(BOR_NEAR_XI, i, x, w);
            const double u = x * umax;
            const double xi = sc * sinh(u);
            const double dx = sc * cosh(u) * w * umax;
            const double s = sin(0.5 * xi);
            const double R = sqrt(r0 * r0 + rr4 * s * s);
            double sk, ck;
            sincos(k * R, &sk, &ck);
            const double f = dx / (4.0 * GRIM_PI * R);
            sg[i] = make_double2(ck * f, -sk * f);
            scos[i] = xi;
        }
        __syncthreads();
        if (t < nm) {
            for (int i = 0; i < BOR_NEAR_XI; ++i) {
                const double c2 = cos(t * scos[i]);
                gsum.x += sg[i].x * c2;
                gsum.y += sg[i].y * c2;
            }
            sG[t] = gsum;
        }
        __syncthreads();
    }
    if (t < nm) {
        const double2 g = sG[t];
        const double ww = p.w * q.w, rr = p.rho * q.rho * ww;
        const double Ta[2] = {p.T0, p.T1}, Da[2] = {p.D0, p.D1};
        const double Tc[2] = {q.T0, q.T1}, Dc[2] = {q.D0, q.D1};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int s = 2 * a + cc;
                const double fa = Ta[a] * Tc[cc] * rr, fdd = Da[a] * Dc[cc] * ww, fdt = Da[a] * Tc[cc] * ww,
                             ftd = Ta[a] * Dc[cc] * ww, ftt = Ta[a] * Tc[cc] * ww;
                acc[s].x += fa * g.x;        acc[s].y += fa * g.y;
                acc[4 + s].x += fdd * g.x;   acc[4 + s].y += fdd * g.y;
                acc[8 + s].x += fdt * g.x;   acc[8 + s].y += fdt * g.y;
                acc[12 + s].x += ftd * g.x;  acc[12 + s].y += ftd * g.y;
                acc[16 + s].x += ftt * g.x;  acc[16 + s].y += ftt * g.y;
            }
    }
}

// grid = (ne, ne); dynamic smem: nxi_cap * (16 + 8) bytes + BOR_MAX_MODES * 16.
__global__ void __launch_bounds__(128)
k_bor_moments(int ne, const double *__restrict__ nodes, double k, int mmax, int nxi_cap, double2 *__restrict__ mom) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // layout sized by the host for nxi_cap samples: sg[nxi_cap], scos[nxi_cap], sG[BOR_MAX_MODES]
    double2 *sg = reinterpret_cast<double2 *>(smem_raw);
    double *scos = reinterpret_cast<double *>(sg + nxi_cap);
    double2 *sG = reinterpret_cast<double2 *>(scos + nxi_cap);
    const int e = blockIdx.x, f = blockIdx.y;
    const int nm = mmax + 2;
    const bool near = abs(e - f) <= 1;
    double2 acc[BOR_SLOTS];
#pragma unroll
    for (int s = 0; s < BOR_SLOTS; ++s) acc[s] = make_double2(0.0, 0.0);
    for (int ip = 0; ip < BOR_FAR_ORDER; ++ip) {
        double xo, wo;
        gl_node(BOR_FAR_ORDER, ip, xo, wo);
        const double so = 0.5 * (xo + 1.0);
        const BorPt p = bor_point(nodes, e, so, 0.5 * wo);
        if (!near) {
            for (int iq = 0; iq < BOR_FAR_ORDER; ++iq) {
                double xs, wsq;
                gl_node(BOR_FAR_ORDER, iq, xs, wsq);
                const BorPt q = bor_point(nodes, f, 0.5 * (xs + 1.0), 0.5 * wsq);
                bor_pair_accumulate(k, p, q, false, mmax, nxi_cap, sg, scos, sG, acc);
            }
        } else {
            const int nq = (e == f) ? 2 * BOR_NEAR_ORDER : BOR_NEAR_ORDER;
            for (int iq = 0; iq < nq; ++iq) {
                double s, ws;
                near_src(e, f, so, iq, s, ws);
                const BorPt q = bor_point(nodes, f, s, ws);
                bor_pair_accumulate(k, p, q, true, mmax, nxi_cap, sg, scos, sG, acc);
            }
        }
    }
    if (threadIdx.x < nm) {
        double2 *o = mom + (((int64_t)e * ne + f) * nm + threadIdx.x) * BOR_SLOTS;
#pragma unroll
        for (int s = 0; s < BOR_SLOTS; ++s) o[s] = acc[s];
    }
}

// grid = ceil(nred / 16) x ceil(nred / 16), block 16 x 16.  rmap[2*nn] gives, for every
// full component index (t: node, phi: nn + node), the reduced index or -1; tie[2*nn]
// holds the complex weight of that component inside its reduced function (1 or
// j m sign(t_rho) for a pole phi folded into the pole t function).  For each reduced
// pair, the entry is sum over full components mapping to it of conj(w_row) Z_full w_col.
// full2red: for reduced index r, up to two full components (f0, f1) with weights.
__global__ void k_bor_assemble(int ne, int mmax, int m, double k, const double2 *__restrict__ mom, int nred,
                               const int *__restrict__ red_full, const double2 *__restrict__ red_w,
                               const double *__restrict__ nodes, double2 *__restrict__ Z, int64_t ldz) {
    const int r = blockIdx.x * 16 + threadIdx.x;  // row (test)
    const int c = blockIdx.y * 16 + threadIdx.y;  // column (source)
    if (r >= nred || c >= nred) return;
    const int nn = ne + 1;
    const int nm = mmax + 2;
    const int am = abs(m), am1 = abs(m - 1), ap1 = abs(m + 1);
    const double km2 = 1.0 / (k * k);
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
            double2 z = make_double2(0.0, 0.0);
            // element pairs (e, f) with e in {ni-1, ni}, f in {nj-1, nj}
            for (int de = 0; de < 2; ++de) {
                const int e = ni - 1 + de;
                if (e < 0 || e >= ne) continue;
                const int a = 1 - de;  // node ni is node index a of element e (e = ni-1 -> a = 1)
                const double tre = (nodes[2 * e + 2] - nodes[2 * e]) /
                                   hypot(nodes[2 * e + 2] - nodes[2 * e], nodes[2 * e + 3] - nodes[2 * e + 1]);
                const double tze = (nodes[2 * e + 3] - nodes[2 * e + 1]) /
                                   hypot(nodes[2 * e + 2] - nodes[2 * e], nodes[2 * e + 3] - nodes[2 * e + 1]);
                for (int df = 0; df < 2; ++df) {
                    const int f = nj - 1 + df;
                    if (f < 0 || f >= ne) continue;
                    const int b = 1 - df;
                    const double trf = (nodes[2 * f + 2] - nodes[2 * f]) /
                                       hypot(nodes[2 * f + 2] - nodes[2 * f], nodes[2 * f + 3] - nodes[2 * f + 1]);
                    const double tzf = (nodes[2 * f + 3] - nodes[2 * f + 1]) /
                                       hypot(nodes[2 * f + 2] - nodes[2 * f], nodes[2 * f + 3] - nodes[2 * f + 1]);
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
                }
            }
            // conj(wr) * z * wc
            const double2 t1 = make_double2(wr.x * z.x + wr.y * z.y, wr.x * z.y - wr.y * z.x);
            total.x += t1.x * wc.x - t1.y * wc.y;
            total.y += t1.x * wc.y + t1.y * wc.x;
        }
    }
    // scale j k eta 2 pi
    const double s = k * 376.730313668 * 2.0 * GRIM_PI;
    Z[(int64_t)c * ldz + r] = make_double2(-s * total.y, s * total.x);
}

// J_m(x) for any integer m (J_{-m} = (-1)^m J_m), through CUDA's jn.
__device__ __forceinline__ double jn_signed(int m, double x) {
    if (x == 0.0) return m == 0 ? 1.0 : 0.0;  // on-axis aspects: J_n(0) = delta_n0
    if (m >= 0) return jn(m, x);
    const double v = jn(-m, x);
    return ((-m) & 1) ? -v : v;
}

// Reduced excitation (far = 0) or far-field weights (far = 1) for mode m.
// Columns: [VV theta_0..n-1, HH theta_0..n-1].  One thread per (reduced row, column).
__global__ void k_bor_excitation(int ne, const double *__restrict__ nodes, double k, int m, int nth,
                                 const double *__restrict__ th_deg, int far, int nred, const int *__restrict__ red_full,
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
            const double r0 = nodes[2 * e], z0 = nodes[2 * e + 1], dr = nodes[2 * e + 2] - r0, dz = nodes[2 * e + 3] - z0;
            const double L = hypot(dr, dz), tr = dr / L, tz = dz / L;
            for (int ip = 0; ip < BOR_FAR_ORDER; ++ip) {
                double xg, wg;
                gl_node(BOR_FAR_ORDER, ip, xg, wg);
                const double s = 0.5 * (xg + 1.0);
                const double rho = r0 + s * dr, z = z0 + s * dz, w = 0.5 * wg * L;
                const double T = a == 0 ? 1.0 - s : s;
                const double x = k * rho * st;
                const double jm = jn_signed(m, x), jm1 = jn_signed(m - 1, x), jp1 = jn_signed(m + 1, x);
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
                double sp, cp;
                sincos(k * z * ct, &sp, &cp);
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
