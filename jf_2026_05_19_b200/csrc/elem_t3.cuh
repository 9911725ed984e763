// elem_t3.cuh -- CTRIA3 stiffness (K) and differential stiffness (KG) kernels.
//
// K: one warp per element.  stiffness_tria3_matrices_generic
// (src/FEMKernels.jl:7315-7385): CST membrane, plate block from the three
// virtual quads of tria3_plate_macro_data (:7157-7209) -- each the plate
// part (bending with twist correction + MacNeal shear, no bending
// incompatible modes) of a default-kwarg stiffness_quad4_matrices -- summed
// into a 21x21 system whose 12 internal dofs are condensed by an LU solve,
// plus the centroidal Hughes-Brezzi drill; then T'KT (assembly.jl:3866-3955).
//
// KG: one thread per element.  CST membrane resultant of stress_strain_tria3
// (FEMKernels.jl:7391-7404) and geometric_stiffness_tria3's non-curvature
// branch (:8083-8097), which the default principal-transverse mode falls
// into; T'KgT and drill zeroing as in assembly.jl:6019-6157.
#pragma once
#include "elem_q4.cuh"

namespace jfg {

constexpr int T3_WARPS = 4;
constexpr int T3_THREADS = 32 * T3_WARPS;

__constant__ int c_t3_quads[3][4] = {{0, 3, 6, 5}, {1, 4, 6, 3}, {2, 5, 6, 4}};

struct T3KShared {
    double p[3][3];
    double v[3][3];
    double lc[3][2];
    double Q[3][9];
    double pts[7][2];
    double bv[3], cv[3], A;
    double Cm[9], Cb[9], Cs[4], h, alpha_d;
    int plate, skip_macneal;
    double dNx[3][5][4], dNy[3][5][4], wdet[3][4];
    double D[3][4][12], Jp[3][4], Zinv[3][16], Y[3][4][12];
    double K[21][22];     // padded row stride
    double X[12][9];      // condensation right-hand side / solution
    int piv;
};

__global__ void __launch_bounds__(T3_THREADS) t3_k_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                         const double *__restrict__ prop,
                                                         const double *__restrict__ coords,
                                                         const double *__restrict__ nodeR, double k6rot, ElemOut o) {
    __shared__ T3KShared sh[T3_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * T3_WARPS + warp;
    if (e >= nt) return;  // whole warp exits together
    T3KShared &S = sh[warp];
    int32_t nd[3];
    for (int k = 0; k < 3; ++k) nd[k] = __ldg(nodes + 3 * e + k);
    if (lane < 3) {
        for (int i = 0; i < 3; ++i) S.p[lane][i] = __ldg(coords + 3 * (int64_t)nd[lane] + i);
    }
    __syncwarp();
    if (lane == 0) {
        double v1[3], v2[3], v3[3];
        t3_frame(S.p[0], S.p[1], S.p[2], v1, v2, v3);
        double c[3];
        for (int i = 0; i < 3; ++i) c[i] = (S.p[0][i] + S.p[1][i] + S.p[2][i]) / 3.0;
        for (int k = 0; k < 3; ++k) {
            double d[3];
            sub3(S.p[k], c, d);
            S.lc[k][0] = dot3(d, v1);
            S.lc[k][1] = dot3(d, v2);
        }
        for (int i = 0; i < 3; ++i) { S.v[0][i] = v1[i]; S.v[1][i] = v2[i]; S.v[2][i] = v3[i]; }
        double x[3] = {S.lc[0][0], S.lc[1][0], S.lc[2][0]}, y[3] = {S.lc[0][1], S.lc[1][1], S.lc[2][1]};
        double A2 = x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]);
        double A = 0.5 * fabs(A2);
        S.A = A;
        S.bv[0] = (y[1] - y[2]) / (2 * A); S.bv[1] = (y[2] - y[0]) / (2 * A); S.bv[2] = (y[0] - y[1]) / (2 * A);
        S.cv[0] = (x[2] - x[1]) / (2 * A); S.cv[1] = (x[0] - x[2]) / (2 * A); S.cv[2] = (x[1] - x[0]) / (2 * A);
        for (int i = 0; i < 3; ++i) { S.pts[i][0] = x[i]; S.pts[i][1] = y[i]; }
        S.pts[3][0] = (x[0] + x[1]) / 2; S.pts[3][1] = (y[0] + y[1]) / 2;
        S.pts[4][0] = (x[1] + x[2]) / 2; S.pts[4][1] = (y[1] + y[2]) / 2;
        S.pts[5][0] = (x[2] + x[0]) / 2; S.pts[5][1] = (y[2] + y[0]) / 2;
        S.pts[6][0] = (x[0] + x[1] + x[2]) / 3; S.pts[6][1] = (y[0] + y[1] + y[2]) / 3;
        const double *pr = prop + 7 * e;
        double h = __ldg(pr), E = __ldg(pr + 1), nu = __ldg(pr + 2), br = __ldg(pr + 4), tst = __ldg(pr + 5), Gs = __ldg(pr + 6);
        double cm = E * h / (1 - nu * nu);
        double cb = br * (E * h * h * h) / (12 * (1 - nu * nu));
        double base[9] = {1.0, nu, 0.0, nu, 1.0, 0.0, 0.0, 0.0, (1 - nu) / 2};
        for (int i = 0; i < 9; ++i) { S.Cm[i] = cm * base[i]; S.Cb[i] = cb * base[i]; }
        bool membrane_only = br <= 1e-12;
        double cs = membrane_only ? 0.0 : tst * h * Gs;
        S.Cs[0] = cs; S.Cs[1] = 0.0; S.Cs[2] = 0.0; S.Cs[3] = cs;
        S.h = h;
        S.plate = (!membrane_only && A >= 1e-12) ? 1 : 0;
        S.skip_macneal = (h < 1e-30 || fabs(cs) < 1e-30) ? 1 : 0;
        double k6 = membrane_only ? 0.0 : k6rot;
        S.alpha_d = (k6 / 1e5) * Gs * h;  // G_ref = shear-material G (assembly.jl:2468)
    }
    __syncwarp();
    const bool degenerate = S.A < 1e-12;
    if (lane < 3) {
        const double *R = nodeR ? nodeR + 9 * (int64_t)nd[lane] : nullptr;
        double Rl[9];
        if (R)
            for (int i = 0; i < 9; ++i) Rl[i] = __ldg(R + i);
        node_block(S.v[0], S.v[1], S.v[2], R ? Rl : nullptr, S.Q[lane]);
    }
    if (S.plate) {
        // virtual-quad Jacobians: lanes 3..17 -> (quad q, point g)
        if (lane >= 3 && lane < 18) {
            int q = (lane - 3) / 5, g = (lane - 3) % 5;
            double lq[4][2];
            for (int k = 0; k < 4; ++k) { lq[k][0] = S.pts[c_t3_quads[q][k]][0]; lq[k][1] = S.pts[c_t3_quads[q][k]][1]; }
            double r = 0.0, s = 0.0;
            if (g < 4) q4_shape_gp(g, r, s);
            double dNr[4] = {-0.25 * (1 - s), 0.25 * (1 - s), 0.25 * (1 + s), -0.25 * (1 + s)};
            double dNs[4] = {-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r), 0.25 * (1 - r)};
            double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
            for (int k = 0; k < 4; ++k) {
                J11 += dNr[k] * lq[k][0]; J12 += dNr[k] * lq[k][1];
                J21 += dNs[k] * lq[k][0]; J22 += dNs[k] * lq[k][1];
            }
            double det = J11 * J22 - J12 * J21;
            double inv = 1.0 / det;
            double iJ11 = J22 * inv, iJ12 = -J12 * inv, iJ21 = -J21 * inv, iJ22 = J11 * inv;
            for (int k = 0; k < 4; ++k) {
                S.dNx[q][g][k] = iJ11 * dNr[k] + iJ12 * dNs[k];
                S.dNy[q][g][k] = iJ21 * dNr[k] + iJ22 * dNs[k];
            }
            if (g < 4) { double a = fabs(det); S.wdet[q][g] = a < 1e-12 ? 1e-12 : a; }
        } else if (lane >= 18 && lane < 30) {
            // MacNeal strain-sampling rows: (quad q, sample point sp)
            int q = (lane - 18) >> 2, sp = (lane - 18) & 3;
            double lq[4][2];
            for (int k = 0; k < 4; ++k) { lq[k][0] = S.pts[c_t3_quads[q][k]][0]; lq[k][1] = S.pts[c_t3_quads[q][k]][1]; }
            const double pt = 0.57735026918962576451;
            const double xs[4] = {0.0, 0.0, -pt, pt}, es[4] = {-pt, pt, 0.0, 0.0};
            double xi = xs[sp], eta = es[sp];
            double dNr[4] = {-0.25 * (1 - eta), 0.25 * (1 - eta), 0.25 * (1 + eta), -0.25 * (1 + eta)};
            double dNs[4] = {-0.25 * (1 - xi), -0.25 * (1 + xi), 0.25 * (1 + xi), 0.25 * (1 - xi)};
            double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
            for (int k = 0; k < 4; ++k) {
                J11 += dNr[k] * lq[k][0]; J12 += dNr[k] * lq[k][1];
                J21 += dNs[k] * lq[k][0]; J22 += dNs[k] * lq[k][1];
            }
            double det = J11 * J22 - J12 * J21;
            if (fabs(det) < 1e-14) det = det < 0.0 ? -1e-14 : 1e-14;
            S.Jp[q][sp] = fabs(det);
            double inv = 1.0 / det;
            double iJ11 = J22 * inv, iJ12 = -J12 * inv, iJ21 = -J21 * inv, iJ22 = J11 * inv;
            for (int k = 0; k < 4; ++k) {
                double dx = iJ11 * dNr[k] + iJ12 * dNs[k], dy = iJ21 * dNr[k] + iJ22 * dNs[k];
                double Nk = 0.25 * (1 + ((k == 1 || k == 2) ? xi : -xi)) * (1 + (k >= 2 ? eta : -eta));
                if (sp < 2) { S.D[q][sp][3 * k] = dx; S.D[q][sp][3 * k + 1] = 0.0; S.D[q][sp][3 * k + 2] = Nk; }
                else { S.D[q][sp][3 * k] = dy; S.D[q][sp][3 * k + 1] = -Nk; S.D[q][sp][3 * k + 2] = 0.0; }
            }
        }
        for (int i = lane; i < 21 * 22; i += 32) (&S.K[0][0])[i] = 0.0;
    }
    __syncwarp();
    if (S.plate && !S.skip_macneal && lane < 3) {
        const int q = lane;
        double lq[4][2];
        for (int k = 0; k < 4; ++k) { lq[k][0] = S.pts[c_t3_quads[q][k]][0]; lq[k][1] = S.pts[c_t3_quads[q][k]][1]; }
        double Dx = 0.5 * (lq[1][0] + lq[2][0] - lq[0][0] - lq[3][0]);
        double Dy = 0.5 * (lq[2][1] + lq[3][1] - lq[0][1] - lq[1][1]);
        double Dx2 = Dx * Dx, Dy2 = Dy * Dy;
        double J11c = 0.25 * (-lq[0][0] + lq[1][0] + lq[2][0] - lq[3][0]);
        double J12c = 0.25 * (-lq[0][1] + lq[1][1] + lq[2][1] - lq[3][1]);
        double J21c = 0.25 * (-lq[0][0] - lq[1][0] + lq[2][0] + lq[3][0]);
        double J22c = 0.25 * (-lq[0][1] - lq[1][1] + lq[2][1] + lq[3][1]);
        double A_elem = 4.0 * fabs(J11c * J22c - J12c * J21c);
        const double eps = 0.04;
        double ap = eps / (eps + (1.0 - eps) * Dx2 / fmax(Dy2, 1e-30));
        double bp = eps / (eps + (1.0 - eps) * Dy2 / fmax(Dx2, 1e-30));
        double flex_x = 1.0 / fmax(fabs(S.Cb[0]), 1e-30), flex_y = 1.0 / fmax(fabs(S.Cb[4]), 1e-30);
        double inv12A = 1.0 / (12.0 * A_elem);
        const double zb = 0.65;
        double zxu = zb * inv12A * Dx2 * flex_x, zxd = zb * inv12A * ap * Dx2 * flex_x;
        double zyu = zb * inv12A * Dy2 * flex_y, zyd = zb * inv12A * bp * Dy2 * flex_y;
        double Zb[16] = {zxu + zxd, zxu - zxd, 0, 0, zxu - zxd, zxu + zxd, 0, 0,
                         0, 0, zyu + zyd, zyu - zyd, 0, 0, zyu - zyd, zyu + zyd};
        double VGV[16];
        const int comps[4] = {1, 1, 2, 2};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                double Jf = sqrt(2.0 * S.Jp[q][i]) * sqrt(2.0 * S.Jp[q][j]);
                double v;
                if (comps[i] == comps[j]) v = (i == j) ? Jf * (comps[i] == 1 ? S.Cs[0] : S.Cs[3]) : 0.0;
                else v = 0.5 * Jf * S.Cs[1];
                VGV[4 * i + j] = v;
            }
        for (int i = 0; i < 4; ++i)
            if (VGV[5 * i] < 1e-30) VGV[5 * i] = 1e-30;
        double Zs[16];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) Zs[4 * i + j] = 0.5 * (VGV[4 * i + j] + VGV[4 * j + i]);
        inv4_inplace(Zs);
        double Zt[16];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) Zt[4 * i + j] = 0.5 * (Zs[4 * i + j] + Zs[4 * j + i]) + Zb[4 * i + j];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) S.Zinv[q][4 * i + j] = 0.5 * (Zt[4 * i + j] + Zt[4 * j + i]);
        inv4_inplace(S.Zinv[q]);
    }
    __syncwarp();
    if (S.plate && !S.skip_macneal) {
        for (int w = lane; w < 144; w += 32) {
            int q = w / 48, l = (w % 48) / 12, j = w % 12;
            double s = 0.0;
            for (int m = 0; m < 4; ++m) s += S.Zinv[q][4 * l + m] * S.D[q][m][j];
            S.Y[q][l][j] = s;
        }
    }
    __syncwarp();
    // plate blocks of the three virtual quads into the 21x21 system
    if (S.plate) {
        for (int q = 0; q < 3; ++q) {
            for (int w = lane; w < 144; w += 32) {
                int i = w / 12, j = w % 12;       // plate index: node i/3, comp i%3 (w, theta_x, theta_y)
                int ka = i / 3, ca = i % 3, kb = j / 3, cb = j % 3;
                double v = 0.0;
                if (ca > 0 && cb > 0) {
                    for (int g = 0; g < 4; ++g) {
                        double a[3], b[3];
                        double xa = S.dNx[q][g][ka], ya = S.dNy[q][g][ka], xb = S.dNx[q][g][kb], yb = S.dNy[q][g][kb];
                        if (ca == 1) { a[0] = 0.0; a[1] = -ya; a[2] = 2.0 * (-xa) - (-S.dNx[q][4][ka]); }
                        else { a[0] = xa; a[1] = 0.0; a[2] = 2.0 * ya - S.dNy[q][4][ka]; }
                        if (cb == 1) { b[0] = 0.0; b[1] = -yb; b[2] = 2.0 * (-xb) - (-S.dNx[q][4][kb]); }
                        else { b[0] = xb; b[1] = 0.0; b[2] = 2.0 * yb - S.dNy[q][4][kb]; }
                        v += S.wdet[q][g] * quad_form(a, S.Cb, b);
                    }
                }
                if (!S.skip_macneal) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int l = 0; l < 4; ++l) {
                        s1 += S.D[q][l][i] * S.Y[q][l][j];
                        s2 += S.D[q][l][j] * S.Y[q][l][i];
                    }
                    v += 0.5 * (s1 + s2);
                }
                int ri = 3 * c_t3_quads[q][ka] + ca, rj = 3 * c_t3_quads[q][kb] + cb;
                S.K[ri][rj] += v;
            }
            __syncwarp();
        }
        // condensation: solve Kii X = Kie (12 x 12, 9 rhs), partial pivoting
        for (int w = lane; w < 108; w += 32) S.X[w / 9][w % 9] = S.K[9 + w / 9][w % 9];
        __syncwarp();
        for (int k = 0; k < 12; ++k) {
            if (lane == 0) {
                int p = k;
                double best = fabs(S.K[9 + k][9 + k]);
                for (int i = k + 1; i < 12; ++i) {
                    double v = fabs(S.K[9 + i][9 + k]);
                    if (v > best) { best = v; p = i; }
                }
                S.piv = p;
            }
            __syncwarp();
            int p = S.piv;
            if (p != k) {
                if (lane < 12) { double t = S.K[9 + k][9 + lane]; S.K[9 + k][9 + lane] = S.K[9 + p][9 + lane]; S.K[9 + p][9 + lane] = t; }
                else if (lane < 21) { int j = lane - 12; double t = S.X[k][j]; S.X[k][j] = S.X[p][j]; S.X[p][j] = t; }
            }
            __syncwarp();
            const double pivv = S.K[9 + k][9 + k];
            // rows i > k: factor and update (lanes over (i, column) items)
            const int nr = 11 - k;
            for (int w = lane; w < nr * 22; w += 32) {
                int i = k + 1 + w / 22, j = w % 22;
                double f = S.K[9 + i][9 + k] / pivv;
                if (j < 12) { if (j > k) S.K[9 + i][9 + j] -= f * S.K[9 + k][9 + j]; }
                else if (j < 21) S.X[i][j - 12] -= f * S.X[k][j - 12];
            }
            __syncwarp();
        }
        // back substitution, one lane per right-hand side column
        if (lane < 9) {
            for (int k = 11; k >= 0; --k) {
                double s = S.X[k][lane];
                for (int i = k + 1; i < 12; ++i) s -= S.K[9 + k][9 + i] * S.X[i][lane];
                S.X[k][lane] = s / S.K[9 + k][9 + k];
            }
        }
        __syncwarp();
        // Kcond = Kee + Kei * Aint,  Aint = -X   (stored back into K[0:9][0:9])
        double kc[3];
        int cnt = 0;
        for (int w = lane; w < 81; w += 32) {
            int i = w / 9, j = w % 9;
            double s = S.K[i][j];
            for (int l = 0; l < 12; ++l) s -= S.K[i][9 + l] * S.X[l][j];
            kc[cnt++] = s;
        }
        __syncwarp();
        cnt = 0;
        for (int w = lane; w < 81; w += 32) S.K[w / 9][w % 9] = kc[cnt++];
        __syncwarp();
    }
    // node-pair sub-blocks: lane -> (pair 0..5, sub-block tt, tr, rt, rr)
    double lmax = 0.0;
    if (lane < 24) {
        const int pr_a[6] = {0, 0, 0, 1, 1, 2}, pr_b[6] = {0, 1, 2, 1, 2, 2};
        const int pair = lane >> 2, sub = lane & 3;
        const int a = pr_a[pair], b = pr_b[pair];
        const int bi = sub >> 1, bj = sub & 1;
        double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (!degenerate) {
            const double A = S.A;
            // membrane CST (u, v) and drill (u, v, theta_z) terms
            double Bd_a[6] = {0.5 * S.cv[a], -0.5 * S.bv[a], 0, 0, 0, 1.0 / 3.0};
            double Bd_b[6] = {0.5 * S.cv[b], -0.5 * S.bv[b], 0, 0, 0, 1.0 / 3.0};
            double ma[2][3] = {{S.bv[a], 0.0, S.cv[a]}, {0.0, S.cv[a], S.bv[a]}};
            double mb[2][3] = {{S.bv[b], 0.0, S.cv[b]}, {0.0, S.cv[b], S.bv[b]}};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    int gi = 3 * bi + i, gj = 3 * bj + j;  // local dof index 0..5
                    double v = S.alpha_d * (Bd_a[gi] * Bd_b[gj]) * A;
                    if (gi < 2 && gj < 2) v += quad_form(ma[gi], S.Cm, mb[gj]) * A;
                    // plate (w, theta_x, theta_y) = local 2, 3, 4
                    if (S.plate && gi >= 2 && gi <= 4 && gj >= 2 && gj <= 4) v += S.K[3 * a + gi - 2][3 * b + gj - 2];
                    L[i][j] = v;
                }
        }
        double O[3][3];
        rot_block(S.Q[a], L, S.Q[b], O);
        const int32_t s = __ldg(o.blk_slot + e * 6 + pair);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double v = O[i][j];
                lmax = fmax(lmax, fabs(v));
                *blk_entry(o, s, 3 * bi + i, 3 * bj + j) = v;
                if (o.diag_staging && a == b && bi == bj && i == j)
                    o.diag_staging[__ldg(o.diag_slot + e * 18 + 6 * a + 3 * bi + i)] = v;
            }
    }
    if (o.maxabs) {
        for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
        if (lane == 0 && lmax > 0.0) atomic_max_nonneg(o.maxabs, lmax);
    }
}

__global__ void __launch_bounds__(128) t3_kg_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                   const double *__restrict__ prop,
                                                   const double *__restrict__ coords,
                                                   const double *__restrict__ nodeR,
                                                   const double *__restrict__ u, ElemOut o) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nt) return;
    int32_t nd[3];
    double p[3][3];
    for (int k = 0; k < 3; ++k) {
        nd[k] = __ldg(nodes + 3 * e + k);
        for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
    }
    double v1[3], v2[3], v3[3];
    t3_frame(p[0], p[1], p[2], v1, v2, v3);
    double c[3], lc[3][2];
    for (int i = 0; i < 3; ++i) c[i] = (p[0][i] + p[1][i] + p[2][i]) / 3.0;
    for (int k = 0; k < 3; ++k) {
        double d[3];
        sub3(p[k], c, d);
        lc[k][0] = dot3(d, v1);
        lc[k][1] = dot3(d, v2);
    }
    double Q[3][9];
    for (int k = 0; k < 3; ++k) {
        double Rl[9];
        if (nodeR)
            for (int i = 0; i < 9; ++i) Rl[i] = __ldg(nodeR + 9 * (int64_t)nd[k] + i);
        node_block(v1, v2, v3, nodeR ? Rl : nullptr, Q[k]);
    }
    const double *pr = prop + 7 * e;
    const double h = __ldg(pr), E = __ldg(pr + 1), nu = __ldg(pr + 2);
    double x[3] = {lc[0][0], lc[1][0], lc[2][0]}, y[3] = {lc[0][1], lc[1][1], lc[2][1]};
    double A = 0.5 * fabs(x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]));
    double val[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (A >= 1e-12 && h >= 1e-30) {
        double b[3] = {(y[1] - y[2]) / (2 * A), (y[2] - y[0]) / (2 * A), (y[0] - y[1]) / (2 * A)};
        double cv[3] = {(x[2] - x[1]) / (2 * A), (x[0] - x[2]) / (2 * A), (x[1] - x[0]) / (2 * A)};
        double eps0 = 0.0, eps1 = 0.0, eps2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double *ug = u + 6 * (int64_t)nd[k];
            double u0 = __ldg(ug), u1 = __ldg(ug + 1), u2 = __ldg(ug + 2);
            double ul = Q[k][0] * u0 + Q[k][1] * u1 + Q[k][2] * u2;
            double vl = Q[k][3] * u0 + Q[k][4] * u1 + Q[k][5] * u2;
            eps0 += b[k] * ul;
            eps1 += cv[k] * vl;
            eps2 += cv[k] * ul + b[k] * vl;
        }
        double cm = E / (1 - nu * nu);
        double Nx = (cm * eps0 + cm * nu * eps1) * h;
        double Ny = (cm * nu * eps0 + cm * eps1) * h;
        double Nxy = (cm * (1 - nu) / 2 * eps2) * h;
        double sxx = Nx / h, syy = Ny / h, sxy = Nxy / h;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                val[i][j] = h * A * (sxx * b[i] * b[j] + syy * cv[i] * cv[j] + sxy * (b[i] * cv[j] + cv[i] * b[j]));
    }
    int pair = 0;
    for (int a = 0; a < 3; ++a)
        for (int bb = a; bb < 3; ++bb, ++pair) {
            double L[3][3] = {{val[a][bb], 0, 0}, {0, val[a][bb], 0}, {0, 0, val[a][bb]}};
            double O[3][3];
            rot_block(Q[a], L, Q[bb], O);
            const int32_t s = __ldg(o.blk_slot + e * 6 + pair);
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) *blk_entry(o, s, i, j) = (i < 3 && j < 3) ? O[i][j] : 0.0;
        }
}

}  // namespace jfg
