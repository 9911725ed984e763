// elem_dkdh.cuh -- shell-thickness sensitivities of the element stiffness.
//
// The reference differentiates stiffness_quad4_generic / stiffness_tria3_generic
// (src/FEMKernels.jl:1473-1656, :7113-7123) in the shell thickness h by
// forward-mode AD (src/solver/dKdx.jl:218-250) and uses dK_e/dh through
//   pseudo-load   sum_e T_e' dK_e/dh T_e u_e        (_scatter_elem_contribution!)
//   contractions  a_e' T_e' dK_e/dh T_e b_e          (compliance / buckling
//                                                      sensitivities per element)
// CQUAD4: the generic element is membrane (Wilson modes condensed), bending
// without the twist row, drilling and tied transverse shear scaled by phi2.
// Cm, K_ab, K_bb and the drill scale are linear in h, Cb cubic, the shear
// linear times phi2 = 10 h^2 / L^2 (or 1 once saturated), so
//   dK/dh = (Km + Kd - Kc + 3 Kb + s Ks) / h,  s = 3 (phi2 < 1) or 1.
// One thread per element forms the strains of a and b (or u) at the Gauss
// points, so no 24x24 matrix is built: a contraction is a sum of strain
// products, a pseudo-load a sum of B' (C strain) terms.
#pragma once
#include "elem_t3.cuh"

namespace jfg {

// Local element vector x_loc = T x_elem of a CQUAD4 (node blocks Q_k, both
// the translation and the rotation triple).
__device__ __forceinline__ void q4_gather_local(const double *__restrict__ xg, const int nd[4], const double Q[4][9],
                                                double xl[24]) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const double *p = xg + 6 * (int64_t)nd[k] + 3 * half;
            const double x0 = __ldg(p), x1 = __ldg(p + 1), x2 = __ldg(p + 2);
#pragma unroll
            for (int r = 0; r < 3; ++r) xl[6 * k + 3 * half + r] = Q[k][3 * r] * x0 + Q[k][3 * r + 1] * x1 + Q[k][3 * r + 2] * x2;
        }
}

// Geometry of the generic CQUAD4 at one Gauss point.
struct Q4GenGp {
    double dx[4], dy[4], N[4], wd, iJ[4], d1x, d1y, d2x, d2y, wem, wep, wxm, wxp;
};

__device__ __forceinline__ void q4_gen_gp(const double lc[4][2], int g, Q4GenGp &G) {
    double r, s;
    q4_shape_gp(g, r, s);
    const double det = q4_point_derivs(lc, r, s, false, G.dx, G.dy, G.iJ);
    const double a = fabs(det);
    G.wd = a < 1e-12 ? 1e-12 : a;
#pragma unroll
    for (int k = 0; k < 4; ++k) G.N[k] = q4_N(k, r, s);
    G.d1x = G.iJ[0] * (-2.0 * r); G.d1y = G.iJ[2] * (-2.0 * r);
    G.d2x = G.iJ[1] * (-2.0 * s); G.d2y = G.iJ[3] * (-2.0 * s);
    G.wem = 0.5 * (1.0 - s); G.wep = 0.5 * (1.0 + s); G.wxm = 0.5 * (1.0 - r); G.wxp = 0.5 * (1.0 + r);
}

// Tied shear rows: tying point t in {(0,-1), (0,1), (-1,0), (1,0)} gives
// coefficients of (w, theta_x, theta_y) of each node (FEMKernels.jl:1510-1538).
struct Q4Tying { double cw[4][4], cx[4][4], cy[4][4]; };

__device__ __forceinline__ void q4_tying(const double lc[4][2], Q4Tying &T) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const double xi = t < 2 ? 0.0 : (t == 2 ? -1.0 : 1.0), eta = t < 2 ? (t == 0 ? -1.0 : 1.0) : 0.0;
        const double dNr[4] = {-0.25 * (1 - eta), 0.25 * (1 - eta), 0.25 * (1 + eta), -0.25 * (1 + eta)};
        const double dNs[4] = {-0.25 * (1 - xi), -0.25 * (1 + xi), 0.25 * (1 + xi), 0.25 * (1 - xi)};
        double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            J11 += dNr[k] * lc[k][0]; J12 += dNr[k] * lc[k][1];
            J21 += dNs[k] * lc[k][0]; J22 += dNs[k] * lc[k][1];
        }
        const double N[4] = {0.25 * (1.0 - xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 + eta),
                             0.25 * (1.0 - xi) * (1.0 + eta)};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            T.cw[t][k] = t < 2 ? dNr[k] : dNs[k];
            T.cx[t][k] = -(t < 2 ? J12 : J22) * N[k];
            T.cy[t][k] = (t < 2 ? J11 : J21) * N[k];
        }
    }
}

// Strains of a local element vector x at a Gauss point: membrane (3),
// curvature without twist row (3), drill (1).
struct Q4Strain { double em[3], kb[3], d; };

__device__ __forceinline__ void q4_gen_strain(const Q4GenGp &G, const double x[24], Q4Strain &S) {
    S.em[0] = S.em[1] = S.em[2] = S.kb[0] = S.kb[1] = S.kb[2] = S.d = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double u = x[6 * k], v = x[6 * k + 1], tx = x[6 * k + 3], ty = x[6 * k + 4], tz = x[6 * k + 5];
        S.em[0] += G.dx[k] * u; S.em[1] += G.dy[k] * v; S.em[2] += G.dy[k] * u + G.dx[k] * v;
        S.kb[0] += G.dx[k] * ty; S.kb[1] -= G.dy[k] * tx; S.kb[2] += G.dy[k] * ty - G.dx[k] * tx;
        S.d += 0.5 * G.dy[k] * u - 0.5 * G.dx[k] * v + G.N[k] * tz;
    }
}

// Tied shear values of x at the four tying points.
__device__ __forceinline__ void q4_tying_values(const Q4Tying &T, const double x[24], double tp[4]) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) s += T.cw[t][k] * x[6 * k + 2] + T.cx[t][k] * x[6 * k + 3] + T.cy[t][k] * x[6 * k + 4];
        tp[t] = s;
    }
}

// e' P(nu) f for the plane-stress base matrix P = [1 nu 0; nu 1 0; 0 0 (1-nu)/2].
__device__ __forceinline__ double pform(const double e[3], const double f[3], double nu, double gam) {
    return e[0] * f[0] + nu * (e[0] * f[1] + e[1] * f[0]) + e[1] * f[1] + gam * e[2] * f[2];
}

// Incompatible-mode loads Bi' sigma (4).
__device__ __forceinline__ void q4_bi_t(const Q4GenGp &G, const double sg[3], double out[4]) {
    out[0] = G.d1x * sg[0] + G.d1y * sg[2];
    out[1] = G.d1y * sg[1] + G.d1x * sg[2];
    out[2] = G.d2x * sg[0] + G.d2y * sg[2];
    out[3] = G.d2y * sg[1] + G.d2x * sg[2];
}

struct Q4GenScalars {
    double h, nu, gam, cm, cb, cs, ad, phi2, sfac;
};

__device__ __forceinline__ Q4GenScalars q4_gen_scalars(const double lc[4][2], double h, double E, double nu) {
    Q4GenScalars c;
    c.h = h; c.nu = nu; c.gam = (1 - nu) / 2;
    c.cm = E * h / (1 - nu * nu);
    c.cb = 1.0 * (E * h * h * h) / (12 * (1 - nu * nu));
    const double G = E / (2 * (1 + nu));
    c.cs = (5.0 / 6.0) * G * h;
    c.ad = (100.0 / 1e5) * G * h;
    const double J11c = 0.25 * (-lc[0][0] + lc[1][0] + lc[2][0] - lc[3][0]);
    const double J12c = 0.25 * (-lc[0][1] + lc[1][1] + lc[2][1] - lc[3][1]);
    const double J21c = 0.25 * (-lc[0][0] - lc[1][0] + lc[2][0] + lc[3][0]);
    const double J22c = 0.25 * (-lc[0][1] - lc[1][1] + lc[2][1] + lc[3][1]);
    const double L2 = fmax(4.0 * fabs(J11c * J22c - J12c * J21c), 1e-30);
    const double trial = 10.0 * h * h / L2;
    c.phi2 = trial < 1.0 ? trial : 1.0;
    c.sfac = trial < 1.0 ? 3.0 : 1.0;
    return c;
}

// Membrane incompatible-mode matrix K_bb / cm (packed upper triangle),
// accumulated with the Gauss-point weight.
__device__ __forceinline__ void q4_bb_add(const Q4GenGp &G, double nu, double gam, double B[10]) {
    const double d1x = G.d1x, d1y = G.d1y, d2x = G.d2x, d2y = G.d2y, wd = G.wd;
    const double P[4][3] = {{d1x, nu * d1x, gam * d1y}, {nu * d1y, d1y, gam * d1x}, {d2x, nu * d2x, gam * d2y}, {nu * d2y, d2y, gam * d2x}};
    B[0] += wd * (d1x * P[0][0] + d1y * P[0][2]);
    B[1] += wd * (d1x * P[1][0] + d1y * P[1][2]);
    B[2] += wd * (d1x * P[2][0] + d1y * P[2][2]);
    B[3] += wd * (d1x * P[3][0] + d1y * P[3][2]);
    B[4] += wd * (d1y * P[1][1] + d1x * P[1][2]);
    B[5] += wd * (d1y * P[2][1] + d1x * P[2][2]);
    B[6] += wd * (d1y * P[3][1] + d1x * P[3][2]);
    B[7] += wd * (d2x * P[2][0] + d2y * P[2][2]);
    B[8] += wd * (d2x * P[3][0] + d2y * P[3][2]);
    B[9] += wd * (d2y * P[3][1] + d2x * P[3][2]);
}

// Element setup shared by both CQUAD4 modes: nodes, frame, local
// coordinates, node blocks.
__device__ __forceinline__ void q4_dkdh_setup(int64_t e, const int32_t *__restrict__ nodes, const double *__restrict__ coords,
                                              const double *__restrict__ nodeR, int nd[4], double lc[4][2], double Q[4][9]) {
    double p[4][3], V[9];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        nd[k] = __ldg(nodes + 4 * e + k);
#pragma unroll
        for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
    }
    q4_local(p, V, lc);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (nodeR) {
            double R[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) R[i] = __ldg(nodeR + 9 * (int64_t)nd[k] + i);
            node_block(V, V + 3, V + 6, R, Q[k]);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) Q[k][i] = V[i];
        }
    }
}

// Thickness derivative (times h) of MacNeal's shear term of node pair (a, b)
// of one virtual quad, added to P: M = D' Z^-1 D with Z = Zs + Zb, where
// Zs = diag(1/vd) goes as 1/h (vd ~ cs ~ h) and Zb as 1/cb ~ h^-3, so
//   h dM/dh = Y' (Zs + 3 Zb) Y,   Y = Z^-1 D = W D.
// Z, W and Zs + 3 Zb are block diagonal (xi rows 0-1, eta rows 2-3), and
// D's columns are: w -> (dN/dx on xi rows, dN/dy on eta rows), theta_x ->
// -N on the eta rows, theta_y -> N on the xi rows.
__device__ __forceinline__ void macneal_dpair(const double (*Dd)[4], const double *W, const double *ivd, const double *zs,
                                              int a, int b, double P[3][3]) {
    const double pt = 0.57735026918962576451;
    const double zx00 = ivd[0] + 3.0 * zs[0], zx11 = ivd[1] + 3.0 * zs[0], zx01 = 3.0 * zs[1];
    const double zy00 = ivd[2] + 3.0 * zs[2], zy11 = ivd[3] + 3.0 * zs[2], zy01 = 3.0 * zs[3];
    // Y columns of node k: x parts (w, theta_y) and y parts (w, theta_x)
    double xw[2][2], xt[2][2], yw[2][2], yt[2][2];
    const int nk[2] = {a, b};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int k = nk[q];
        const double cx0 = Dd[0][k], cx1 = Dd[1][k], cy0 = Dd[2][k], cy1 = Dd[3][k];
        const double nx0 = q4_N(k, 0.0, -pt), nx1 = q4_N(k, 0.0, pt);
        const double ny0 = -q4_N(k, -pt, 0.0), ny1 = -q4_N(k, pt, 0.0);
        xw[q][0] = W[0] * cx0 + W[1] * cx1; xw[q][1] = W[1] * cx0 + W[2] * cx1;
        xt[q][0] = W[0] * nx0 + W[1] * nx1; xt[q][1] = W[1] * nx0 + W[2] * nx1;
        yw[q][0] = W[3] * cy0 + W[4] * cy1; yw[q][1] = W[4] * cy0 + W[5] * cy1;
        yt[q][0] = W[3] * ny0 + W[4] * ny1; yt[q][1] = W[4] * ny0 + W[5] * ny1;
    }
    auto fx = [&](const double *u, const double *v) { return u[0] * (zx00 * v[0] + zx01 * v[1]) + u[1] * (zx01 * v[0] + zx11 * v[1]); };
    auto fy = [&](const double *u, const double *v) { return u[0] * (zy00 * v[0] + zy01 * v[1]) + u[1] * (zy01 * v[0] + zy11 * v[1]); };
    P[0][0] += fx(xw[0], xw[1]) + fy(yw[0], yw[1]);
    P[0][1] += fy(yw[0], yt[1]);
    P[0][2] += fx(xw[0], xt[1]);
    P[1][0] += fy(yt[0], yw[1]);
    P[1][1] += fy(yt[0], yt[1]);
    P[2][0] += fx(xt[0], xw[1]);
    P[2][2] += fx(xt[0], xt[1]);
}

// Contractions c[e] = a_e' T' dK/dh T b_e of every CQUAD4.
__global__ void __launch_bounds__(128) q4_dkdh_contract_kernel(int64_t nq, const int32_t *__restrict__ nodes,
                                                               const double *__restrict__ prop,
                                                               const double *__restrict__ coords,
                                                               const double *__restrict__ nodeR,
                                                               const double *__restrict__ a, const double *__restrict__ b,
                                                               double *c) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nq) return;
    int nd[4];
    double lc[4][2], Q[4][9];
    q4_dkdh_setup(e, nodes, coords, nodeR, nd, lc, Q);
    const double *pr = prop + 7 * e;
    const Q4GenScalars C = q4_gen_scalars(lc, __ldg(pr), __ldg(pr + 1), __ldg(pr + 2));
    double al[24], bl[24];
    q4_gather_local(a, nd, Q, al);
    q4_gather_local(b, nd, Q, bl);
    Q4Tying T;
    q4_tying(lc, T);
    double ta[4], tb[4];
    q4_tying_values(T, al, ta);
    q4_tying_values(T, bl, tb);
    double qm = 0.0, qb = 0.0, qd = 0.0, qs = 0.0, ka[4] = {0, 0, 0, 0}, kb[4] = {0, 0, 0, 0};
    double B[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
        Q4GenGp G;
        q4_gen_gp(lc, g, G);
        Q4Strain Sa, Sb;
        q4_gen_strain(G, al, Sa);
        q4_gen_strain(G, bl, Sb);
        qm += G.wd * pform(Sa.em, Sb.em, C.nu, C.gam);
        qb += G.wd * pform(Sa.kb, Sb.kb, C.nu, C.gam);
        qd += G.wd * (Sa.d * Sb.d);
        const double ga[2] = {G.wem * ta[0] + G.wep * ta[1], G.wxm * ta[2] + G.wxp * ta[3]};
        const double gb[2] = {G.wem * tb[0] + G.wep * tb[1], G.wxm * tb[2] + G.wxp * tb[3]};
        // gamma_a' invJ' invJ gamma_b
        const double xa0 = G.iJ[0] * ga[0] + G.iJ[1] * ga[1], xa1 = G.iJ[2] * ga[0] + G.iJ[3] * ga[1];
        const double xb0 = G.iJ[0] * gb[0] + G.iJ[1] * gb[1], xb1 = G.iJ[2] * gb[0] + G.iJ[3] * gb[1];
        qs += G.wd * (xa0 * xb0 + xa1 * xb1);
        // K_ab' x / cm: membrane stresses of x against the incompatible modes
        const double sa[3] = {Sa.em[0] + C.nu * Sa.em[1], C.nu * Sa.em[0] + Sa.em[1], C.gam * Sa.em[2]};
        const double sb[3] = {Sb.em[0] + C.nu * Sb.em[1], C.nu * Sb.em[0] + Sb.em[1], C.gam * Sb.em[2]};
        double ia[4], ib[4];
        q4_bi_t(G, sa, ia);
        q4_bi_t(G, sb, ib);
#pragma unroll
        for (int l = 0; l < 4; ++l) { ka[l] += G.wd * ia[l]; kb[l] += G.wd * ib[l]; }
        q4_bb_add(G, C.nu, C.gam, B);
    }
    // condensation a' K_ab K_bb^-1 K_ab' b = cm ka' B^-1 kb (K_bb = cm B)
    double qc = 0.0, bmax = 0.0;
#pragma unroll
    for (int i = 0; i < 10; ++i) bmax = fmax(bmax, fabs(B[i]));
    if (bmax * C.cm > 0.0) {
        const Ldl4 f(B);
        double z[4];
        f.solve(kb, z);
        qc = ka[0] * z[0] + ka[1] * z[1] + ka[2] * z[2] + ka[3] * z[3];
    }
    const double km = C.cm * qm, kbv = C.cb * qb, kd = C.ad * qd, ks = C.phi2 * C.cs * qs, kc = C.cm * qc;
    c[e] = (km + kd - kc + 3.0 * kbv + C.sfac * ks) / C.h;
}

// Pseudo-load of the masked CQUAD4 (every CQUAD4 when mask is null):
// f_e = T' dK/dh T u_e, written to the element's dof slots of the diagonal
// staging (slots of unmasked elements keep the zeros the caller put there).
__global__ void __launch_bounds__(128) q4_dkdh_load_kernel(int64_t nq, const int32_t *__restrict__ nodes,
                                                           const double *__restrict__ prop,
                                                           const double *__restrict__ coords,
                                                           const double *__restrict__ nodeR,
                                                           const double *__restrict__ u, const uint8_t *__restrict__ mask,
                                                           const int32_t *__restrict__ dslot, double *stage) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nq || (mask && !__ldg(mask + e))) return;
    int nd[4];
    double lc[4][2], Q[4][9];
    q4_dkdh_setup(e, nodes, coords, nodeR, nd, lc, Q);
    const double *pr = prop + 7 * e;
    const Q4GenScalars C = q4_gen_scalars(lc, __ldg(pr), __ldg(pr + 1), __ldg(pr + 2));
    double ul[24];
    q4_gather_local(u, nd, Q, ul);
    Q4Tying T;
    q4_tying(lc, T);
    double tu[4];
    q4_tying_values(T, ul, tu);
    double f[24];
#pragma unroll
    for (int i = 0; i < 24; ++i) f[i] = 0.0;
    double tw[4] = {0, 0, 0, 0}, ku[4] = {0, 0, 0, 0}, B[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double fm = C.cm, fb = 3.0 * C.cb, fd = C.ad, fs = C.sfac * C.phi2 * C.cs;
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
        Q4GenGp G;
        q4_gen_gp(lc, g, G);
        Q4Strain S;
        q4_gen_strain(G, ul, S);
        const double sm[3] = {S.em[0] + C.nu * S.em[1], C.nu * S.em[0] + S.em[1], C.gam * S.em[2]};
        const double mb[3] = {S.kb[0] + C.nu * S.kb[1], C.nu * S.kb[0] + S.kb[1], C.gam * S.kb[2]};
        const double w = G.wd;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            f[6 * k] += w * (fm * (G.dx[k] * sm[0] + G.dy[k] * sm[2]) + fd * 0.5 * G.dy[k] * S.d);
            f[6 * k + 1] += w * (fm * (G.dy[k] * sm[1] + G.dx[k] * sm[2]) - fd * 0.5 * G.dx[k] * S.d);
            f[6 * k + 3] += w * fb * (-G.dy[k] * mb[1] - G.dx[k] * mb[2]);
            f[6 * k + 4] += w * fb * (G.dx[k] * mb[0] + G.dy[k] * mb[2]);
            f[6 * k + 5] += w * fd * G.N[k] * S.d;
        }
        // tied shear: B_cov' (invJ' invJ) B_cov u, spread back to the tying rows
        const double g0 = G.wem * tu[0] + G.wep * tu[1], g1 = G.wxm * tu[2] + G.wxp * tu[3];
        const double x0 = G.iJ[0] * g0 + G.iJ[1] * g1, x1 = G.iJ[2] * g0 + G.iJ[3] * g1;
        const double h0 = G.iJ[0] * x0 + G.iJ[2] * x1, h1 = G.iJ[1] * x0 + G.iJ[3] * x1;  // invJ' (invJ g)
        tw[0] += w * fs * G.wem * h0; tw[1] += w * fs * G.wep * h0;
        tw[2] += w * fs * G.wxm * h1; tw[3] += w * fs * G.wxp * h1;
        double iu[4];
        q4_bi_t(G, sm, iu);
#pragma unroll
        for (int l = 0; l < 4; ++l) ku[l] += w * iu[l];
        q4_bb_add(G, C.nu, C.gam, B);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            f[6 * k + 2] += tw[t] * T.cw[t][k];
            f[6 * k + 3] += tw[t] * T.cx[t][k];
            f[6 * k + 4] += tw[t] * T.cy[t][k];
        }
    // condensation: - K_ab K_bb^-1 K_ab' u = - cm sum_gp wd Bm' P (Bi z), z = B^-1 ku
    double bmax = 0.0;
#pragma unroll
    for (int i = 0; i < 10; ++i) bmax = fmax(bmax, fabs(B[i]));
    if (bmax * C.cm > 0.0) {
        const Ldl4 fct(B);
        double z[4];
        fct.solve(ku, z);
#pragma unroll 1
        for (int g = 0; g < 4; ++g) {
            Q4GenGp G;
            q4_gen_gp(lc, g, G);
            const double ei[3] = {G.d1x * z[0] + G.d2x * z[2], G.d1y * z[1] + G.d2y * z[3],
                                  G.d1y * z[0] + G.d1x * z[1] + G.d2y * z[2] + G.d2x * z[3]};
            const double si[3] = {ei[0] + C.nu * ei[1], C.nu * ei[0] + ei[1], C.gam * ei[2]};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                f[6 * k] -= G.wd * fm * (G.dx[k] * si[0] + G.dy[k] * si[2]);
                f[6 * k + 1] -= G.wd * fm * (G.dy[k] * si[1] + G.dx[k] * si[2]);
            }
        }
    }
    // f_global = T' f_local / h into the element's dof slots
    const double ih = 1.0 / C.h;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int half = 0; half < 2; ++half)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double v = Q[k][c] * f[6 * k + 3 * half] + Q[k][3 + c] * f[6 * k + 3 * half + 1] +
                                 Q[k][6 + c] * f[6 * k + 3 * half + 2];
                stage[__ldg(dslot + 24 * e + 6 * k + 3 * half + c)] = v * ih;
            }
}

// CTRIA3: stiffness_tria3_generic is CST membrane and centroidal drill (both
// linear in h) plus the plate condensed from three MacNeal virtual quads,
// K_c = Kee - Kei X with X = Kii^-1 Kie.  With dK21 the thickness derivative
// of the 21-dof macro plate (3 h dP/dh = 3 K_bend + Y' (Zs + 3 Zb) Y per
// quad), dK_c = [I, -X'] dK21 [I; -X], so a contraction is abar' dK21 bbar
// with xbar = (x_p, -X x_p) and a load is (f_e - X' f_i) with f = dK21 ubar.
// A team of 16 lanes per element, two teams per warp, as in t3_k_kernel.
constexpr int T3D_WARPS = 2;
constexpr int T3D_ELEMS = T3_TEAMS_PER_WARP * T3D_WARPS;

struct T3DShared {
    T3KShared k;
    double dPb[3][10][9];  // h dP/dh per (virtual quad, node pair)
    double vl[2][18];      // local element vectors (a, b; or u)
    double xb[2][21];      // macro-plate vectors: corner dofs 3n + i (n < 3), then -X x_p
    double fb[21];         // load: h dK21/dh ubar
    double fl[18];         // load: h f_local
};

// Node block Q_k = Rel node_R_k of a CTRIA3 node.
__device__ __forceinline__ void t3_node_block(const double V[9], const double *__restrict__ nodeR, int n, double Q[9]) {
    if (nodeR) {
        double R[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) R[i] = __ldg(nodeR + 9 * (int64_t)n + i);
        node_block(V, V + 3, V + 6, R, Q);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) Q[i] = V[i];
    }
}

// LOAD = false: c[e] = a_e' T' dK/dh T b_e of every CTRIA3.
// LOAD = true: f_e = T' dK/dh T u_e of the masked CTRIA3 (all when mask is
// null), written to the element's dof slots of the diagonal staging.
template <bool LOAD>
__global__ void __launch_bounds__(32 * T3D_WARPS) t3_dkdh_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                                 const double *__restrict__ prop,
                                                                 const double *__restrict__ coords,
                                                                 const double *__restrict__ nodeR,
                                                                 const double *__restrict__ va, const double *__restrict__ vb,
                                                                 double *c, const uint8_t *__restrict__ mask,
                                                                 const int32_t *__restrict__ dslot, double *stage) {
    __shared__ T3DShared sh[T3D_ELEMS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane >> 4, tl = lane & 15;
    const unsigned tm = 0xFFFFu << (16 * team);
    const int64_t e = (int64_t)blockIdx.x * T3D_ELEMS + warp * T3_TEAMS_PER_WARP + team;
    if (e >= nt) return;                     // the whole team leaves; syncs below are team-local
    if (LOAD && mask && !__ldg(mask + e)) return;  // the mask is per element, so team-uniform
    T3DShared &D = sh[warp * T3_TEAMS_PER_WARP + team];
    T3KShared &S = D.k;

    // Phase 0, every lane in registers: nodes, corners, frame, local
    // coordinates, generic constitutive scalars (FEMKernels.jl:7113-7123).
    double x[3], y[3], V[9], A, h, nu, gam, cb, cs;
    int nd[3];
    {
        const double *pr = prop + 7 * e;
        h = __ldg(pr);
        const double E = __ldg(pr + 1);
        nu = __ldg(pr + 2);
        double p[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            nd[k] = __ldg(nodes + 3 * e + k);
#pragma unroll
            for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
        }
        double v1[3], v2[3], v3[3];
        t3_frame(p[0], p[1], p[2], v1, v2, v3);
        double cc[3];
        for (int i = 0; i < 3; ++i) cc[i] = (p[0][i] + p[1][i] + p[2][i]) / 3.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double d[3];
            sub3(p[k], cc, d);
            x[k] = dot3(d, v1);
            y[k] = dot3(d, v2);
        }
        for (int i = 0; i < 3; ++i) { V[i] = v1[i]; V[3 + i] = v2[i]; V[6 + i] = v3[i]; }
        A = 0.5 * fabs(x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]));
        gam = (1 - nu) / 2;
        cb = 1.0 * (E * h * h * h / (12 * (1 - nu * nu)));
        const double G = E / (2 * (1 + nu));
        cs = (5.0 / 6.0) * G * h;
        if (tl == 0) {
            const double i2A = 1.0 / (2 * A);
            S.bv[0] = (y[1] - y[2]) * i2A; S.bv[1] = (y[2] - y[0]) * i2A; S.bv[2] = (y[0] - y[1]) * i2A;
            S.cv[0] = (x[2] - x[1]) * i2A; S.cv[1] = (x[0] - x[2]) * i2A; S.cv[2] = (x[1] - x[0]) * i2A;
            S.A = A;
            S.cm = E * h / (1 - nu * nu);
            S.ad = (100.0 / 1e5) * G * h;
        }
    }
    const bool plate = A >= 1e-12, macneal = plate && !(h < 1e-30 || fabs(cs) < 1e-30);
    // local element vectors, entry i = 6 k + 3 half + r
    const int nv = LOAD ? 1 : 2;
    for (int it = tl; it < 18 * nv; it += T3_TEAM) {
        const int v = it / 18, i = it - 18 * v, k = i / 6, half = (i / 3) & 1, r = i % 3;
        const int n = k == 0 ? nd[0] : (k == 1 ? nd[1] : nd[2]);
        const double *xg = (v == 0 ? va : vb) + 6 * (int64_t)n + 3 * half;
        double Q[9];
        t3_node_block(V, nodeR, n, Q);
        D.vl[v][i] = Q[3 * r] * __ldg(xg) + Q[3 * r + 1] * __ldg(xg + 1) + Q[3 * r + 2] * __ldg(xg + 2);
    }
    __syncwarp(tm);

    if (plate) {
        t3_plate_points(S, tl, tm, x, y, cs, cb, macneal);
        // h dP/dh of every (virtual quad, node pair), read before the
        // condensation reuses the quad data's shared memory
        for (int it = tl; it < 30; it += T3_TEAM) {
            const int q = it / 10, pp = it - 10 * q;
            int ka, kb;
            q4_pair(pp, ka, kb);
            double v[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            bend_pair(S.u.q.dNx[q], S.u.q.dNy[q], S.u.q.wdet[q], ka, kb, 3.0 * cb, nu, gam, v);
            if (macneal) macneal_dpair(S.u.q.Dd[q], S.u.q.W[q], S.u.q.ivd[q], S.u.q.zs[q], ka, kb, v);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) D.dPb[q][pp][3 * i + j] = v[i][j];
        }
        t3_plate_blocks(S, tl, tm, cb, nu, gam, macneal);
        t3_condense(S, tl, tm);
        // macro-plate vectors: corner plate dofs, then -X x_p on the internal dofs
        for (int it = tl; it < 21 * nv; it += T3_TEAM) {
            const int v = it / 21, r = it - 21 * v;
            if (r < 9) {
                D.xb[v][r] = D.vl[v][6 * (r / 3) + 2 + r % 3];
            } else {
                double s = 0.0;
#pragma unroll
                for (int cc = 0; cc < 9; ++cc) s += S.u.c.X[r - 9][cc] * D.vl[v][6 * (cc / 3) + 2 + cc % 3];
                D.xb[v][r] = -s;
            }
        }
        __syncwarp(tm);
    }

    if (!LOAD) {
        // abar' (h dK21/dh) bbar: each (virtual quad, node pair) block and its mirror
        double acc = 0.0;
        if (plate) {
            for (int it = tl; it < 30; it += T3_TEAM) {
                const int q = it / 10, pp = it - 10 * q;
                int ka, kb;
                q4_pair(pp, ka, kb);
                const int nA = t3_quad_node(q, ka), nB = t3_quad_node(q, kb);
                const double *P = D.dPb[q][pp];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        acc += D.xb[0][3 * nA + i] * P[3 * i + j] * D.xb[1][3 * nB + j];
                        if (ka != kb) acc += D.xb[0][3 * nB + j] * P[3 * i + j] * D.xb[1][3 * nA + i];
                    }
            }
        }
        for (int off = 8; off > 0; off >>= 1) acc += __shfl_xor_sync(tm, acc, off, 16);
        if (tl == 0) {
            double cmd = 0.0;
            if (A >= 1e-12) {
                // CST membrane and centroidal drill, both linear in h
                double ea[3] = {0, 0, 0}, eb[3] = {0, 0, 0}, da = 0.0, db = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double bk = S.bv[k], ck = S.cv[k];
                    const double ua = D.vl[0][6 * k], wa = D.vl[0][6 * k + 1], ub = D.vl[1][6 * k], wb = D.vl[1][6 * k + 1];
                    ea[0] += bk * ua; ea[1] += ck * wa; ea[2] += ck * ua + bk * wa;
                    eb[0] += bk * ub; eb[1] += ck * wb; eb[2] += ck * ub + bk * wb;
                    da += 0.5 * ck * ua - 0.5 * bk * wa + (1.0 / 3.0) * D.vl[0][6 * k + 5];
                    db += 0.5 * ck * ub - 0.5 * bk * wb + (1.0 / 3.0) * D.vl[1][6 * k + 5];
                }
                cmd = (S.cm * pform(ea, eb, nu, gam)) * S.A + S.ad * (da * db) * S.A;
            }
            c[e] = (cmd + acc) / h;
        }
        return;
    }

    if (plate) {
        // fbar = (h dK21/dh) ubar, one macro-plate dof per item
        for (int it = tl; it < 21; it += T3_TEAM) {
            const int n = it / 3, i = it - 3 * n;
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int la = 0; la < 4; ++la) {
                    if (t3_quad_node(q, la) != n) continue;
#pragma unroll
                    for (int kb = 0; kb < 4; ++kb) {
                        const int nB = t3_quad_node(q, kb);
                        const bool tr = la > kb;
                        const int pid = tr ? packed_index(kb, la, 4) : packed_index(la, kb, 4);
#pragma unroll
                        for (int j = 0; j < 3; ++j) s += D.dPb[q][pid][tr ? 3 * j + i : 3 * i + j] * D.xb[0][3 * nB + j];
                    }
                }
            D.fb[it] = s;
        }
        __syncwarp(tm);
    }
    // h f_local: plate rows (corner part minus X' internal part), membrane and drill rows
    for (int it = tl; it < 18; it += T3_TEAM) {
        const int k = it / 6, dof = it - 6 * k;
        double f = 0.0;
        if (A >= 1e-12) {
            if (dof >= 2 && dof <= 4) {
                if (plate) {
                    const int ci = 3 * k + dof - 2;
                    f = D.fb[ci];
                    for (int r = 0; r < 12; ++r) f -= S.u.c.X[r][ci] * D.fb[9 + r];
                }
            } else {
                double ep[3] = {0, 0, 0}, dd = 0.0;
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    const double bm = S.bv[m], cm_ = S.cv[m], uu = D.vl[0][6 * m], vv = D.vl[0][6 * m + 1];
                    ep[0] += bm * uu; ep[1] += cm_ * vv; ep[2] += cm_ * uu + bm * vv;
                    dd += 0.5 * cm_ * uu - 0.5 * bm * vv + (1.0 / 3.0) * D.vl[0][6 * m + 5];
                }
                const double s0 = S.cm * (ep[0] + nu * ep[1]), s1 = S.cm * (nu * ep[0] + ep[1]), s2 = S.cm * (gam * ep[2]);
                const double bk = S.bv[k], ck = S.cv[k];
                if (dof == 0) f = S.A * (bk * s0 + ck * s2) + S.ad * S.A * (0.5 * ck) * dd;
                else if (dof == 1) f = S.A * (ck * s1 + bk * s2) + S.ad * S.A * (-0.5 * bk) * dd;
                else f = S.ad * S.A * (1.0 / 3.0) * dd;
            }
        }
        D.fl[it] = f;
    }
    __syncwarp(tm);
    // f_global = T' f_local / h into the element's dof slots
    for (int it = tl; it < 18; it += T3_TEAM) {
        const int k = it / 6, half = (it / 3) & 1, cc = it % 3;
        const int n = k == 0 ? nd[0] : (k == 1 ? nd[1] : nd[2]);
        double Q[9];
        t3_node_block(V, nodeR, n, Q);
        const double *fl = D.fl + 6 * k + 3 * half;
        stage[__ldg(dslot + 18 * e + it)] = (Q[cc] * fl[0] + Q[3 + cc] * fl[1] + Q[6 + cc] * fl[2]) / h;
    }
}

// Per-element a_e' KG_e b_e from the staged KG blocks of one shell type (the
// KG element kernels' output before the reduction; the element matrices of
// the KG assembly before constraints).  NN nodes, NN(NN+1)/2 node pairs per
// element in slot-map order; a regular slot holds the translation 3x3 in
// stored orientation, an RBE2-path pair its raw 6x6 block.  With a = b = phi
// this is phi' KG_e phi, and divided by h_e the thickness sensitivity of
// _dKg_dx_phi_thickness (src/solver/adjoint_buckling.jl:2079-2150): KG is
// linear in h at fixed u.
template <int NN>
__global__ void __launch_bounds__(128) kg_contract_kernel(int64_t ne, const int32_t *__restrict__ nodes,
                                                          const int32_t *__restrict__ blk_slot,
                                                          const double *__restrict__ staging,
                                                          const double *__restrict__ exc_raw,
                                                          const double *__restrict__ a, const double *__restrict__ b,
                                                          double *__restrict__ c) {
    constexpr int NP = NN * (NN + 1) / 2;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int32_t nd[NN];
#pragma unroll
    for (int k = 0; k < NN; ++k) nd[k] = __ldg(nodes + NN * e + k);
    double s = 0.0;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        int pa, pb;
        if (NN == 4) {
            q4_pair(p, pa, pb);
        } else {
            pa = (p >= 3) + (p >= 5);
            pb = pa + p - (pa == 0 ? 0 : (pa == 1 ? 3 : 5));
        }
        const int32_t sl = __ldg(blk_slot + NP * e + p);
        const double *ua = a + 6 * (int64_t)nd[pa], *ub = b + 6 * (int64_t)nd[pb];
        const double *va = a + 6 * (int64_t)nd[pb], *vb = b + 6 * (int64_t)nd[pa];
        if (sl >= 0) {
            const double *S = staging + 12 * (int64_t)(sl & kBlkIndexMask);
            const bool t = sl & kBlkTranspose;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double g = t ? __ldg(S + 3 * j + i) : __ldg(S + 3 * i + j);
                    s += __ldg(ua + i) * g * __ldg(ub + j);
                    if (pa != pb) s += __ldg(va + j) * g * __ldg(vb + i);
                }
        } else {
            const double *R = exc_raw + 36 * (int64_t)(-(sl + 1));
#pragma unroll
            for (int i = 0; i < 6; ++i)
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    const double g = __ldg(R + 6 * i + j);
                    s += __ldg(ua + i) * g * __ldg(ub + j);
                    if (pa != pb) s += __ldg(va + j) * g * __ldg(vb + i);
                }
        }
    }
    c[e] = s;
}

}  // namespace jfg
