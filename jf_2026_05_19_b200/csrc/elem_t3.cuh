// elem_t3.cuh -- CTRIA3 stiffness (K) and differential stiffness (KG) kernels.
//
// K: a team of 16 lanes per element, two teams per warp; each team
// synchronises only its own lanes.  stiffness_tria3_matrices_generic
// (src/FEMKernels.jl:7315-7385): CST membrane, plate block from the three
// virtual quads of tria3_plate_macro_data (:7157-7209) -- each the plate
// part (bending with twist correction + MacNeal shear, no bending
// incompatible modes) of a default-kwarg stiffness_quad4_matrices -- summed
// into a 21x21 system whose 12 internal dofs are condensed, plus the
// centroidal Hughes-Brezzi drill; then T'KT (assembly.jl:3866-3955).
//
// Macro nodes: corners 0-2, edge midpoints 3 (0-1), 4 (1-2), 5 (2-0),
// centroid 6.  No virtual quad holds two corners, so Kee is block diagonal
// and every Kei entry comes from the one quad that holds the corner.  The
// internal solve lu(Kii) \ Kie runs as Gauss-Jordan elimination with one row
// of [Kii | Kie] per lane in registers: pivot choice, row positions and the
// forward elimination are those of LU with partial pivoting (max |a_ik|,
// first position on ties); eliminating above the pivot as well replaces the
// back substitution.
//
// KG: one thread per (element, node pair).  CST membrane resultant of stress_strain_tria3
// (FEMKernels.jl:7391-7404) and geometric_stiffness_tria3's non-curvature
// branch (:8083-8097), which the default principal-transverse mode falls
// into; T'KgT and drill zeroing as in assembly.jl:6019-6157.
#pragma once
#include "elem_q4.cuh"

namespace jfg {

constexpr int T3_TEAM = 16;
constexpr int T3_TEAMS_PER_WARP = 2;
constexpr int T3_WARPS = 4;
constexpr int T3_THREADS = 32 * T3_WARPS;
constexpr int T3_ELEMS_PER_BLOCK = T3_TEAMS_PER_WARP * T3_WARPS;

// virtual quads of tria3_plate_macro_data (TRIA3_MACRO_QUADS), macro node ids
__host__ __device__ constexpr int t3_quad_node(int q, int k) {
    return q == 0 ? (k == 0 ? 0 : k == 1 ? 3 : k == 2 ? 6 : 5)
         : q == 1 ? (k == 0 ? 1 : k == 1 ? 4 : k == 2 ? 6 : 3)
                  : (k == 0 ? 2 : k == 1 ? 5 : k == 2 ? 6 : 4);
}
__constant__ int c_t3_quads[3][4] = {{0, 3, 6, 5}, {1, 4, 6, 3}, {2, 5, 6, 4}};

struct T3KShared {
    double p[3][3];
    double v[3][3];
    double Q[3][9];
    double pts[7][2];
    double bv[3], cv[3], A;
    double Cm[9], Cb[9], cs, alpha_d;
    int nd[3], plate, skip_macneal;
    union {
        struct {  // virtual-quad data (phases 2-4)
            double dNx[3][5][4], dNy[3][5][4], wdet[3][4];
            double D[3][4][12], Jp[3][4];
            MacNealZ mz[3];
        } q;
        struct {  // condensation (phases 5-7)
            double X[12][9];
            double Kc[9][9];
        } c;
    } u;
    double Pb[3][10][9];  // quad q, local node pair (a <= b): 3x3 over (w, theta_x, theta_y)
};

__global__ void __launch_bounds__(T3_THREADS, 5) t3_k_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                         const double *__restrict__ prop,
                                                         const double *__restrict__ coords,
                                                         const double *__restrict__ nodeR, double k6rot, ElemOut o) {
    __shared__ T3KShared sh[T3_ELEMS_PER_BLOCK];
    o = o.at(blockIdx.y);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane >> 4, tl = lane & 15;
    const unsigned tm = 0xFFFFu << (16 * team);
    const int64_t e = (int64_t)blockIdx.x * T3_ELEMS_PER_BLOCK + warp * T3_TEAMS_PER_WARP + team;
    if (e >= nt) return;  // the whole team leaves; syncs below are team-local
    T3KShared &S = sh[warp * T3_TEAMS_PER_WARP + team];

    // Phase 0: connectivity and coordinates; the property record is loaded
    // now so that its latency overlaps the coordinate loads.
    double h = 0.0, E = 0.0, nu = 0.0, br = 0.0, tst = 0.0, Gs = 0.0;
    if (tl == 0) {
        const double *pr = prop + 7 * e;
        h = o.thickness(e, pr); E = __ldg(pr + 1); nu = __ldg(pr + 2); br = __ldg(pr + 4); tst = __ldg(pr + 5);
        Gs = __ldg(pr + 6);
    }
    if (tl < 3) {
        const int32_t n = __ldg(nodes + 3 * e + tl);
        S.nd[tl] = n;
        for (int i = 0; i < 3; ++i) S.p[tl][i] = __ldg(coords + 3 * (int64_t)n + i);
    }
    __syncwarp(tm);
    // Phase 1: frame, macro points, constitutive data (one lane).
    if (tl == 0) {
        double v1[3], v2[3], v3[3];
        t3_frame(S.p[0], S.p[1], S.p[2], v1, v2, v3);
        double c[3], lc[3][2];
        for (int i = 0; i < 3; ++i) c[i] = (S.p[0][i] + S.p[1][i] + S.p[2][i]) / 3.0;
        for (int k = 0; k < 3; ++k) {
            double d[3];
            sub3(S.p[k], c, d);
            lc[k][0] = dot3(d, v1);
            lc[k][1] = dot3(d, v2);
        }
        for (int i = 0; i < 3; ++i) { S.v[0][i] = v1[i]; S.v[1][i] = v2[i]; S.v[2][i] = v3[i]; }
        double x[3] = {lc[0][0], lc[1][0], lc[2][0]}, y[3] = {lc[0][1], lc[1][1], lc[2][1]};
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
        double cm = E * h / (1 - nu * nu);
        double cb = br * (E * h * h * h) / (12 * (1 - nu * nu));
        double base[9] = {1.0, nu, 0.0, nu, 1.0, 0.0, 0.0, 0.0, (1 - nu) / 2};
        for (int i = 0; i < 9; ++i) { S.Cm[i] = cm * base[i]; S.Cb[i] = cb * base[i]; }
        bool membrane_only = br <= 1e-12;
        double cs = membrane_only ? 0.0 : tst * h * Gs;
        S.cs = cs;
        S.plate = (!membrane_only && A >= 1e-12) ? 1 : 0;
        S.skip_macneal = (h < 1e-30 || fabs(cs) < 1e-30) ? 1 : 0;
        double k6 = membrane_only ? 0.0 : k6rot;
        S.alpha_d = (k6 / 1e5) * Gs * h;  // G_ref = shear-material G (assembly.jl:2468)
    }
    __syncwarp(tm);
    const bool plate = S.plate != 0, macneal = plate && !S.skip_macneal;

    // Phase 2: node blocks (items 0-2), virtual-quad Jacobians (3-17) and
    // MacNeal strain-sampling rows (18-29), two items per lane.
    for (int it = tl; it < 30; it += T3_TEAM) {
        if (it < 3) {
            const double *R = nodeR ? nodeR + 9 * (int64_t)S.nd[it] : nullptr;
            double Rl[9];
            if (R)
                for (int i = 0; i < 9; ++i) Rl[i] = __ldg(R + i);
            node_block(S.v[0], S.v[1], S.v[2], R ? Rl : nullptr, S.Q[it]);
        } else if (!plate) {
        } else if (it < 18) {
            int q = (it - 3) / 5, g = (it - 3) % 5;
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
                S.u.q.dNx[q][g][k] = iJ11 * dNr[k] + iJ12 * dNs[k];
                S.u.q.dNy[q][g][k] = iJ21 * dNr[k] + iJ22 * dNs[k];
            }
            if (g < 4) { double a = fabs(det); S.u.q.wdet[q][g] = a < 1e-12 ? 1e-12 : a; }
        } else {
            int q = (it - 18) >> 2, sp = (it - 18) & 3;
            double lq[4][2];
            for (int k = 0; k < 4; ++k) { lq[k][0] = S.pts[c_t3_quads[q][k]][0]; lq[k][1] = S.pts[c_t3_quads[q][k]][1]; }
            const double pt = 0.57735026918962576451;
            double xi = sp < 2 ? 0.0 : (sp == 2 ? -pt : pt), eta = sp >= 2 ? 0.0 : (sp == 0 ? -pt : pt);
            double dNr[4] = {-0.25 * (1 - eta), 0.25 * (1 - eta), 0.25 * (1 + eta), -0.25 * (1 + eta)};
            double dNs[4] = {-0.25 * (1 - xi), -0.25 * (1 + xi), 0.25 * (1 + xi), 0.25 * (1 - xi)};
            double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
            for (int k = 0; k < 4; ++k) {
                J11 += dNr[k] * lq[k][0]; J12 += dNr[k] * lq[k][1];
                J21 += dNs[k] * lq[k][0]; J22 += dNs[k] * lq[k][1];
            }
            double det = J11 * J22 - J12 * J21;
            if (fabs(det) < 1e-14) det = det < 0.0 ? -1e-14 : 1e-14;
            S.u.q.Jp[q][sp] = fabs(det);
            double inv = 1.0 / det;
            double iJ11 = J22 * inv, iJ12 = -J12 * inv, iJ21 = -J21 * inv, iJ22 = J11 * inv;
            for (int k = 0; k < 4; ++k) {
                double dx = iJ11 * dNr[k] + iJ12 * dNs[k], dy = iJ21 * dNr[k] + iJ22 * dNs[k];
                double Nk = 0.25 * (1 + ((k == 1 || k == 2) ? xi : -xi)) * (1 + (k >= 2 ? eta : -eta));
                double *Dr = S.u.q.D[q][sp] + 3 * k;
                if (sp < 2) { Dr[0] = dx; Dr[1] = 0.0; Dr[2] = Nk; }
                else { Dr[0] = dy; Dr[1] = -Nk; Dr[2] = 0.0; }
            }
        }
    }
    __syncwarp(tm);
    // Phase 3: MacNeal compliance factors per virtual quad.
    if (macneal && tl < 3) {
        double lq[4][2];
        for (int k = 0; k < 4; ++k) { lq[k][0] = S.pts[c_t3_quads[tl][k]][0]; lq[k][1] = S.pts[c_t3_quads[tl][k]][1]; }
        S.u.q.mz[tl] = macneal_z(lq, S.u.q.Jp[tl], S.cs, S.Cb[0], S.Cb[4]);
    }
    __syncwarp(tm);

    if (plate) {
        // Phase 4: plate 3x3 block of every (virtual quad, node pair).
        for (int it = tl; it < 30; it += T3_TEAM) {
            const int q = it / 10, pp = it - 10 * q;
            const int ka = c_pair_a[pp], kb = c_pair_b[pp];
            double v[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            const double xca = S.u.q.dNx[q][4][ka], yca = S.u.q.dNy[q][4][ka];
            const double xcb = S.u.q.dNx[q][4][kb], ycb = S.u.q.dNy[q][4][kb];
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                const double xa = S.u.q.dNx[q][g][ka], ya = S.u.q.dNy[q][g][ka];
                const double xb = S.u.q.dNx[q][g][kb], yb = S.u.q.dNy[q][g][kb];
                const double wd = S.u.q.wdet[q][g];
                // bending columns (theta_x, theta_y) with the twist correction
                const double ac[2][3] = {{0.0, -ya, 2.0 * (-xa) - (-xca)}, {xa, 0.0, 2.0 * ya - yca}};
                const double bc[2][3] = {{0.0, -yb, 2.0 * (-xb) - (-xcb)}, {xb, 0.0, 2.0 * yb - ycb}};
#pragma unroll
                for (int cj = 0; cj < 2; ++cj) {
                    double cbb[3];
#pragma unroll
                    for (int r = 0; r < 3; ++r)
                        cbb[r] = S.Cb[3 * r] * bc[cj][0] + S.Cb[3 * r + 1] * bc[cj][1] + S.Cb[3 * r + 2] * bc[cj][2];
#pragma unroll
                    for (int ci = 0; ci < 2; ++ci)
                        v[1 + ci][1 + cj] += wd * (ac[ci][0] * cbb[0] + ac[ci][1] * cbb[1] + ac[ci][2] * cbb[2]);
                }
            }
            if (macneal) {
                double Da[4][3], Db[4][3], Ya[4][3], Yb[4][3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    double d[4], y[4];
#pragma unroll
                    for (int l = 0; l < 4; ++l) d[l] = Da[l][c] = S.u.q.D[q][l][3 * ka + c];
                    macneal_y(S.u.q.mz[q], d, y);
#pragma unroll
                    for (int l = 0; l < 4; ++l) Ya[l][c] = y[l];
#pragma unroll
                    for (int l = 0; l < 4; ++l) d[l] = Db[l][c] = S.u.q.D[q][l][3 * kb + c];
                    macneal_y(S.u.q.mz[q], d, y);
#pragma unroll
                    for (int l = 0; l < 4; ++l) Yb[l][c] = y[l];
                }
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        double s1 = 0.0, s2 = 0.0;
#pragma unroll
                        for (int l = 0; l < 4; ++l) {
                            s1 += Da[l][i] * Yb[l][j];
                            s2 += Db[l][j] * Ya[l][i];
                        }
                        v[i][j] += 0.5 * (s1 + s2);
                    }
            }
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) S.Pb[q][pp][3 * i + j] = v[i][j];
        }
        __syncwarp(tm);

        // Phase 5: lane r < 12 holds row r of [Kii | Kie] (internal dof r =
        // macro node 3 + r/3, component r%3), summed over quads in order.
        const bool act = tl < 12;
        const int nA = 3 + tl / 3, ci = tl - 3 * (tl / 3);
        double row[21];
#pragma unroll
        for (int c = 0; c < 21; ++c) row[c] = 0.0;
        if (act) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                int la = -1;
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (t3_quad_node(q, k) == nA) la = k;
                if (la >= 0) {
#pragma unroll
                    for (int kb = 0; kb < 4; ++kb) {
                        const int nB = t3_quad_node(q, kb);
                        const int cb0 = nB >= 3 ? 3 * (nB - 3) : 12 + 3 * nB;
                        const bool tr = la > kb;
                        const int pid = tr ? packed_index(kb, la, 4) : packed_index(la, kb, 4);
#pragma unroll
                        for (int cj = 0; cj < 3; ++cj) row[cb0 + cj] += S.Pb[q][pid][tr ? 3 * cj + ci : 3 * ci + cj];
                    }
                }
            }
        }
        int pos = act ? tl : 64;
        double diag = 1.0;
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const bool cand_ok = act && pos >= k;
            double cv = cand_ok ? fabs(row[k]) : -1.0;
            int cp = cand_ok ? pos : 64;
#pragma unroll
            for (int off = 8; off > 0; off >>= 1) {
                const double ov = __shfl_xor_sync(tm, cv, off, 16);
                const int op = __shfl_xor_sync(tm, cp, off, 16);
                if (ov > cv || (ov == cv && op < cp)) { cv = ov; cp = op; }
            }
            const bool is_piv = act && pos == cp;
            const unsigned bal = __ballot_sync(tm, is_piv) & tm;
            const int src = (__ffs(bal) - 1) & 15;
            if (act && pos == k) pos = cp;  // LU row swap of positions k and cp
            if (is_piv) pos = k;
            const double akk = __shfl_sync(tm, row[k], src, 16);
            if (is_piv) diag = akk;
            const double f = (act && !is_piv) ? row[k] / akk : 0.0;
#pragma unroll
            for (int j = k + 1; j < 21; ++j) {
                const double pj = __shfl_sync(tm, row[j], src, 16);
                row[j] -= f * pj;
            }
        }
        __syncwarp(tm);  // every lane is past its last read of the quad data
        if (act && pos < 12)
#pragma unroll
            for (int c = 0; c < 9; ++c) S.u.c.X[pos][c] = row[12 + c] / diag;
        __syncwarp(tm);

        // Phase 6: Kcond = Kee - Kei X (Kee, Kei from the corner's own quad).
        for (int it = tl; it < 81; it += T3_TEAM) {
            const int r = it / 9, col = it - 9 * r;
            const int c = r / 3, i = r - 3 * c, c2 = col / 3, j = col - 3 * c2;
            double kee = (c == c2) ? S.Pb[c][0][3 * i + j] : 0.0;
            double s = 0.0;
            for (int kl = 1; kl < 4; ++kl) {
                const int l0 = 3 * (c_t3_quads[c][kl] - 3);
#pragma unroll
                for (int lj = 0; lj < 3; ++lj) s += S.Pb[c][kl][3 * i + lj] * S.u.c.X[l0 + lj][col];
            }
            S.u.c.Kc[r][col] = kee - s;
        }
        __syncwarp(tm);
    }

    // Phase 7: node-pair sub-blocks: item -> (pair 0..5, sub-block tt, tr, rt, rr)
    double lmax = 0.0;
    const bool degenerate = S.A < 1e-12;
    for (int it = tl; it < 24; it += T3_TEAM) {
        const int pr_a[6] = {0, 0, 0, 1, 1, 2}, pr_b[6] = {0, 1, 2, 1, 2, 2};
        const int pair = it >> 2, sub = it & 3;
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
                    if (plate && gi >= 2 && gi <= 4 && gj >= 2 && gj <= 4) v += S.u.c.Kc[3 * a + gi - 2][3 * b + gj - 2];
                    L[i][j] = v;
                }
        }
        double O[3][3];
        rot_block(S.Q[a], L, S.Q[b], O);
        const int32_t sl = __ldg(o.blk_slot + e * 6 + pair);
        write_sub_block(o, e, sl, a, b, bi, bj, O, lmax, 18);
    }
    if (o.maxabs) {
        for (int off = 8; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(tm, lmax, off, 16));
        if (tl == 0 && lmax > 0.0) atomic_max_nonneg(o.maxabs, lmax);
    }
}

// One (element, node pair) per thread, laid out pair-major so that a warp
// runs one compile-time pair; each thread recomputes the element's frame and
// membrane stress (cheap) and writes its own pair block.
template <int PA, int PB>
__device__ __forceinline__ void t3_kg_pair(int64_t e, const int32_t *__restrict__ nodes, const double *__restrict__ prop,
                                           const double *__restrict__ coords, const double *__restrict__ nodeR,
                                           const double *__restrict__ u, const ElemOut &o) {
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
    const double h = o.thickness(e, pr), E = __ldg(pr + 1), nu = __ldg(pr + 2);
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
    double L[3][3] = {{val[PA][PB], 0, 0}, {0, val[PA][PB], 0}, {0, 0, val[PA][PB]}};
    double O[3][3];
    rot_block(Q[PA], L, Q[PB], O);
    const int32_t s = __ldg(o.blk_slot + e * 6 + packed_index(PA, PB, 3));
    // staged blocks of KG shells are read as their translation 3x3 only; the
    // dof-level RBE2 path (s < 0) reads whole raw blocks
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j)
            if (i < 3 && j < 3) *blk_entry(o, s, i, j) = O[i][j];
            else if (s < 0) *blk_entry(o, s, i, j) = 0.0;
}

__global__ void __launch_bounds__(128) t3_kg_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                   const double *__restrict__ prop,
                                                   const double *__restrict__ coords,
                                                   const double *__restrict__ nodeR,
                                                   const double *__restrict__ u, ElemOut o) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int pair = (int)(t / nt);
    const int64_t e = t - (int64_t)pair * nt;
    o = o.at(blockIdx.y);
    u += (int64_t)blockIdx.y * o.u_stride;
    switch (pair) {
        case 0: t3_kg_pair<0, 0>(e, nodes, prop, coords, nodeR, u, o); break;
        case 1: t3_kg_pair<0, 1>(e, nodes, prop, coords, nodeR, u, o); break;
        case 2: t3_kg_pair<0, 2>(e, nodes, prop, coords, nodeR, u, o); break;
        case 3: t3_kg_pair<1, 1>(e, nodes, prop, coords, nodeR, u, o); break;
        case 4: t3_kg_pair<1, 2>(e, nodes, prop, coords, nodeR, u, o); break;
        case 5: t3_kg_pair<2, 2>(e, nodes, prop, coords, nodeR, u, o); break;
        default: break;
    }
}

}  // namespace jfg
