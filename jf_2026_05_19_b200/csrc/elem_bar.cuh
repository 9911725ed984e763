// elem_bar.cuh -- CBAR/CBEAM stiffness and differential stiffness kernels.
//
// One thread per element.  K: stiffness_frame3d_generic (Timoshenko frame
// with Cowper shear areas and I12 coupling, src/FEMKernels.jl:140-209) in the
// bar frame of assembly.jl:3961-4025 (offset-aware T with -R*skew(w)*R_node
// blocks), T'kT.  KG: axial force P = (k u_bar)[7] (forces_frame3d,
// FEMKernels.jl:215-229) and the beam-column geometric stiffness
// geometric_stiffness_frame3d (:7441-7471), T'KgT (assembly.jl:6277-6424).
// Bars with offsets never reach the KG kernel: the reference raises on them.
#pragma once
#include "elem_q4.cuh"

namespace jfg {


struct BarFrame {
    double L;
    double Rel[3][3];
    double TR[2][9];     // Rel * node_R for GA, GB
    double Toff[2][9];   // -Rel * skew(w) * node_R, zero without offsets
};

__device__ __forceinline__ bool bar_frame(int64_t e, const int32_t *__restrict__ nodes, const double *__restrict__ prop,
                                          const double *__restrict__ coords, const double *__restrict__ nodeR,
                                          BarFrame &F, int32_t nd[2]) {
    const double *pr = prop + 18 * e;
    nd[0] = __ldg(nodes + 2 * e);
    nd[1] = __ldg(nodes + 2 * e + 1);
    double p1[3], p2[3], wa[3], wb[3];
    for (int i = 0; i < 3; ++i) {
        p1[i] = __ldg(coords + 3 * (int64_t)nd[0] + i);
        p2[i] = __ldg(coords + 3 * (int64_t)nd[1] + i);
        wa[i] = __ldg(pr + 12 + i);
        wb[i] = __ldg(pr + 15 + i);
    }
    bool off = dot3(wa, wa) > 1e-20 || dot3(wb, wb) > 1e-20;
    double a[3], b[3], d[3];
    for (int i = 0; i < 3; ++i) { a[i] = off ? p1[i] + wa[i] : p1[i]; b[i] = off ? p2[i] + wb[i] : p2[i]; }
    sub3(b, a, d);
    F.L = sqrt(dot3(d, d));
    if (F.L < 1e-9) return false;
    double vx[3], vref[3] = {__ldg(pr + 9), __ldg(pr + 10), __ldg(pr + 11)}, t[3], vz[3], vy[3];
    normalize3(d, vx);
    if (sqrt(dot3(vref, vref)) < 1e-6) {
        vref[0] = 0.0; vref[1] = 0.0; vref[2] = 1.0;
        if (fabs(dot3(vx, vref)) > 0.9) { vref[0] = 0.0; vref[1] = 1.0; vref[2] = 0.0; }
    }
    cross3(vx, vref, t);
    normalize3(t, vz);
    cross3(vz, vx, vy);
    for (int i = 0; i < 3; ++i) { F.Rel[0][i] = vx[i]; F.Rel[1][i] = vy[i]; F.Rel[2][i] = vz[i]; }
    for (int k = 0; k < 2; ++k) {
        double R[9];
        if (nodeR) for (int i = 0; i < 9; ++i) R[i] = __ldg(nodeR + 9 * (int64_t)nd[k] + i);
        else for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                F.TR[k][3 * r + c] = F.Rel[r][0] * R[c] + F.Rel[r][1] * R[3 + c] + F.Rel[r][2] * R[6 + c];
        const double *w = k == 0 ? wa : wb;
        if (off) {
            double S[3][3] = {{0.0, -w[2], w[1]}, {w[2], 0.0, -w[0]}, {-w[1], w[0], 0.0}};
            double RS[3][3];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) RS[r][c] = F.Rel[r][0] * S[0][c] + F.Rel[r][1] * S[1][c] + F.Rel[r][2] * S[2][c];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) F.Toff[k][3 * r + c] = -(RS[r][0] * R[c] + RS[r][1] * R[3 + c] + RS[r][2] * R[6 + c]);
        } else {
            for (int i = 0; i < 9; ++i) F.Toff[k][i] = 0.0;
        }
    }
    return true;
}

// T12 entry (row i, col j) from the block structure.
__device__ __forceinline__ double bar_T(const BarFrame &F, int i, int j) {
    int ki = i / 6, kj = j / 6;
    if (ki != kj) return 0.0;
    int ri = i % 6, cj = j % 6;
    if (ri < 3 && cj < 3) return F.TR[ki][3 * ri + cj];
    if (ri >= 3 && cj >= 3) return F.TR[ki][3 * (ri - 3) + cj - 3];
    if (ri < 3 && cj >= 3) return F.Toff[ki][3 * ri + cj - 3];
    return 0.0;
}

__device__ void frame3d_k(const double *__restrict__ pr, double L, double k[12][12]) {
    double A = __ldg(pr), Iz = __ldg(pr + 1), Iy = __ldg(pr + 2), I12 = __ldg(pr + 3), J = __ldg(pr + 4);
    double K1 = __ldg(pr + 5), K2 = __ldg(pr + 6), E = __ldg(pr + 7), G = __ldg(pr + 8);
    if (Iy == 0.0) Iy = Iz;
    if (Iz == 0.0) Iz = Iy;
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) k[i][j] = 0.0;
    double X = E * A / L;
    k[0][0] = X; k[0][6] = -X; k[6][0] = -X; k[6][6] = X;
    double T = G * J / L;
    k[3][3] = T; k[3][9] = -T; k[9][3] = -T; k[9][9] = T;
    bool inf_y = !(K1 > 0.0), inf_z = !(K2 > 0.0);
    double Asy = K1 * A, Asz = K2 * A;
    double Phi_y = inf_z ? 0.0 : 12 * E * Iy / (G * Asz * L * L);
    double Phi_z = inf_y ? 0.0 : 12 * E * Iz / (G * Asy * L * L);
    double a_y = 12 * E * Iy / (L * L * L * (1 + Phi_y)), b_y = 6 * E * Iy / (L * L * (1 + Phi_y));
    double c_y = (4 + Phi_y) * E * Iy / (L * (1 + Phi_y)), d_y = (2 - Phi_y) * E * Iy / (L * (1 + Phi_y));
    k[2][2] = a_y; k[2][8] = -a_y; k[8][2] = -a_y; k[8][8] = a_y;
    k[2][4] = -b_y; k[2][10] = -b_y; k[4][2] = -b_y; k[10][2] = -b_y;
    k[8][4] = b_y; k[8][10] = b_y; k[4][8] = b_y; k[10][8] = b_y;
    k[4][4] = c_y; k[4][10] = d_y; k[10][4] = d_y; k[10][10] = c_y;
    double a_z = 12 * E * Iz / (L * L * L * (1 + Phi_z)), b_z = 6 * E * Iz / (L * L * (1 + Phi_z));
    double c_z = (4 + Phi_z) * E * Iz / (L * (1 + Phi_z)), d_z = (2 - Phi_z) * E * Iz / (L * (1 + Phi_z));
    k[1][1] = a_z; k[1][7] = -a_z; k[7][1] = -a_z; k[7][7] = a_z;
    k[1][5] = b_z; k[1][11] = b_z; k[5][1] = b_z; k[11][1] = b_z;
    k[7][5] = -b_z; k[7][11] = -b_z; k[5][7] = -b_z; k[11][7] = -b_z;
    k[5][5] = c_z; k[5][11] = d_z; k[11][5] = d_z; k[11][11] = c_z;
    if (fabs(I12) > 0.0) {
        double a = 12 * E * I12 / (L * L * L), b = 6 * E * I12 / (L * L), c = 4 * E * I12 / L, d = 2 * E * I12 / L;
        k[1][2] += a; k[2][1] += a; k[1][8] += -a; k[8][1] += -a;
        k[7][2] += -a; k[2][7] += -a; k[7][8] += a; k[8][7] += a;
        k[1][4] += -b; k[4][1] += -b; k[1][10] += -b; k[10][1] += -b;
        k[7][4] += b; k[4][7] += b; k[7][10] += b; k[10][7] += b;
        k[2][5] += b; k[5][2] += b; k[2][11] += b; k[11][2] += b;
        k[8][5] += -b; k[5][8] += -b; k[8][11] += -b; k[11][8] += -b;
        k[4][5] += -c; k[5][4] += -c; k[4][11] += -d; k[11][4] += -d;
        k[10][5] += -d; k[5][10] += -d; k[10][11] += -c; k[11][10] += -c;
    }
}

// Write T' k T (upper triangle) for one bar.
__device__ __forceinline__ void bar_write(const ElemOut &o, int64_t e, const BarFrame &F, const double k[12][12],
                                          const int32_t nd[2], double &lmax) {
    double KT[12][12];
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) {
            double s = 0.0;
            for (int l = 0; l < 12; ++l) s += k[i][l] * bar_T(F, l, j);
            KT[i][j] = s;
        }
    double G[12][12];
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) {
            double s = 0.0;
            for (int l = 0; l < 12; ++l) s += bar_T(F, l, i) * KT[l][j];
            G[i][j] = s;
            lmax = fmax(lmax, fabs(s));
        }
    const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 1};
    for (int p = 0; p < 3; ++p) {
        const int32_t s = __ldg(o.blk_slot + e * 3 + p);
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) *blk_entry(o, s, i, j) = G[6 * pa[p] + i][6 * pb[p] + j];
    }
    if (o.diag_staging)
        for (int i = 0; i < 12; ++i) o.diag_staging[__ldg(o.diag_slot + e * 12 + i)] = G[i][i];
}

__global__ void __launch_bounds__(128) bar_k_kernel(int64_t nb, const int32_t *__restrict__ nodes,
                                                   const double *__restrict__ prop, const double *__restrict__ coords,
                                                   const double *__restrict__ nodeR, ElemOut o) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double lmax = 0.0;
    if (e < nb) {
        BarFrame F;
        int32_t nd[2];
        if (bar_frame(e, nodes, prop, coords, nodeR, F, nd)) {
            double k[12][12];
            frame3d_k(prop + 18 * e, F.L, k);
            bar_write(o, e, F, k, nd, lmax);
        }
    }
    if (o.maxabs) {
        for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
        if ((threadIdx.x & 31) == 0 && lmax > 0.0) atomic_max_nonneg(o.maxabs, lmax);
    }
}

__global__ void __launch_bounds__(128) bar_kg_kernel(int64_t nb, const int32_t *__restrict__ nodes,
                                                    const double *__restrict__ prop, const double *__restrict__ coords,
                                                    const double *__restrict__ nodeR, const double *__restrict__ u,
                                                    ElemOut o) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nb) return;
    BarFrame F;
    int32_t nd[2];
    if (!bar_frame(e, nodes, prop, coords, nodeR, F, nd)) return;
    double ub[12];
    for (int k = 0; k < 2; ++k) {
        double ug[6];
        for (int d = 0; d < 6; ++d) ug[d] = __ldg(u + 6 * (int64_t)nd[k] + d);
        for (int dd = 0; dd < 6; ++dd) {
            double s = 0.0;
            for (int q = 0; q < 6; ++q) s += bar_T(F, 6 * k + dd, 6 * k + q) * ug[q];
            ub[6 * k + dd] = s;
        }
    }
    const double *pr = prop + 18 * e;
    double A = __ldg(pr), E = __ldg(pr + 7);
    double X = E * A / F.L;
    double P = -X * ub[0] + X * ub[6];
    double kg[12][12];
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) kg[i][j] = 0.0;
    double L = F.L;
    if (!(L < 1e-9 || fabs(P) < 1e-30)) {
        double c1 = 6.0 * P / (5.0 * L), c2 = P / 10.0, c3 = 2.0 * P * L / 15.0, c4 = -P * L / 30.0;
        kg[1][1] = c1; kg[7][7] = c1; kg[1][7] = -c1; kg[7][1] = -c1;
        kg[1][5] = c2; kg[5][1] = c2; kg[1][11] = c2; kg[11][1] = c2;
        kg[5][5] = c3; kg[11][11] = c3; kg[5][11] = c4; kg[11][5] = c4;
        kg[7][5] = -c2; kg[5][7] = -c2; kg[7][11] = -c2; kg[11][7] = -c2;
        kg[2][2] = c1; kg[8][8] = c1; kg[2][8] = -c1; kg[8][2] = -c1;
        kg[2][4] = -c2; kg[4][2] = -c2; kg[2][10] = -c2; kg[10][2] = -c2;
        kg[4][4] = c3; kg[10][10] = c3; kg[4][10] = c4; kg[10][4] = c4;
        kg[8][4] = c2; kg[4][8] = c2; kg[8][10] = c2; kg[10][8] = c2;
    }
    double lmax = 0.0;
    bar_write(o, e, F, kg, nd, lmax);
}

}  // namespace jfg
