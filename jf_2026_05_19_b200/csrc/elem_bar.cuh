// elem_bar.cuh -- CBAR/CBEAM stiffness and differential stiffness kernels.
//
// One thread per (element, node pair).  K: stiffness_frame3d_generic (Timoshenko frame
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
    bool off;            // any offset vector nonzero
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
    F.off = off;
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

// Local 12x12 frame matrix of stiffness_frame3d_generic
// (FEMKernels.jl:140-209) or geometric_stiffness_frame3d (:7441-7471) as
// closed-form coefficients.  Dofs per node: u, v, w, theta_x, theta_y,
// theta_z; entry (i, j) is evaluated by frame_k with compile-time indices,
// so the zero pattern folds away and no 12x12 array is formed.
struct FrameK {
    double X, T;               // axial EA/L, torsion GJ/L
    double ay, by, cy, dy;     // bending in the x-z plane (w, theta_y)
    double az, bz, cz, dz;     // bending in the x-y plane (v, theta_z)
    double a12, b12, c12, d12; // I12 coupling (zero when I12 == 0)
};

__device__ __forceinline__ double frame_k(const FrameK &c, int i, int j) {
    const int ni = i / 6, nj = j / 6, li = i % 6, lj = j % 6;
    const bool same = ni == nj;
    if (li == 0 && lj == 0) return same ? c.X : -c.X;
    if (li == 3 && lj == 3) return same ? c.T : -c.T;
    if (li == 2 && lj == 2) return same ? c.ay : -c.ay;
    if (li == 2 && lj == 4) return ni == 0 ? -c.by : c.by;
    if (li == 4 && lj == 2) return nj == 0 ? -c.by : c.by;
    if (li == 4 && lj == 4) return same ? c.cy : c.dy;
    if (li == 1 && lj == 1) return same ? c.az : -c.az;
    if (li == 1 && lj == 5) return ni == 0 ? c.bz : -c.bz;
    if (li == 5 && lj == 1) return nj == 0 ? c.bz : -c.bz;
    if (li == 5 && lj == 5) return same ? c.cz : c.dz;
    if ((li == 1 && lj == 2) || (li == 2 && lj == 1)) return same ? c.a12 : -c.a12;
    if (li == 1 && lj == 4) return ni == 0 ? -c.b12 : c.b12;
    if (li == 4 && lj == 1) return nj == 0 ? -c.b12 : c.b12;
    if (li == 2 && lj == 5) return ni == 0 ? c.b12 : -c.b12;
    if (li == 5 && lj == 2) return nj == 0 ? c.b12 : -c.b12;
    if ((li == 4 && lj == 5) || (li == 5 && lj == 4)) return same ? -c.c12 : -c.d12;
    return 0.0;
}

// Structural nonzeros of the local frame matrix (same pattern as frame_k).
__host__ __device__ constexpr bool frame_nz(int i, int j) {
    return ((i % 6 == 0) && (j % 6 == 0)) || ((i % 6 == 3) && (j % 6 == 3)) ||
           ((i % 6 == 1 || i % 6 == 2 || i % 6 == 4 || i % 6 == 5) && (j % 6 == 1 || j % 6 == 2 || j % 6 == 4 || j % 6 == 5));
}

__device__ __forceinline__ FrameK frame3d_k(const double *__restrict__ pr, double L) {
    double A = __ldg(pr), Iz = __ldg(pr + 1), Iy = __ldg(pr + 2), I12 = __ldg(pr + 3), J = __ldg(pr + 4);
    double K1 = __ldg(pr + 5), K2 = __ldg(pr + 6), E = __ldg(pr + 7), G = __ldg(pr + 8);
    if (Iy == 0.0) Iy = Iz;
    if (Iz == 0.0) Iz = Iy;
    FrameK c;
    c.X = E * A / L;
    c.T = G * J / L;
    bool inf_y = !(K1 > 0.0), inf_z = !(K2 > 0.0);
    double Asy = K1 * A, Asz = K2 * A;
    double Phi_y = inf_z ? 0.0 : 12 * E * Iy / (G * Asz * L * L);
    double Phi_z = inf_y ? 0.0 : 12 * E * Iz / (G * Asy * L * L);
    c.ay = 12 * E * Iy / (L * L * L * (1 + Phi_y)); c.by = 6 * E * Iy / (L * L * (1 + Phi_y));
    c.cy = (4 + Phi_y) * E * Iy / (L * (1 + Phi_y)); c.dy = (2 - Phi_y) * E * Iy / (L * (1 + Phi_y));
    c.az = 12 * E * Iz / (L * L * L * (1 + Phi_z)); c.bz = 6 * E * Iz / (L * L * (1 + Phi_z));
    c.cz = (4 + Phi_z) * E * Iz / (L * (1 + Phi_z)); c.dz = (2 - Phi_z) * E * Iz / (L * (1 + Phi_z));
    if (fabs(I12) > 0.0) {
        c.a12 = 12 * E * I12 / (L * L * L); c.b12 = 6 * E * I12 / (L * L);
        c.c12 = 4 * E * I12 / L; c.d12 = 2 * E * I12 / L;
    } else {
        c.a12 = c.b12 = c.c12 = c.d12 = 0.0;
    }
    return c;
}

// Beam-column geometric stiffness in the same closed form (axial force P).
__device__ __forceinline__ FrameK frame3d_kg(double L, double P) {
    FrameK c;
    c.X = c.T = 0.0;
    c.a12 = c.b12 = c.c12 = c.d12 = 0.0;
    if (L < 1e-9 || fabs(P) < 1e-30) {
        c.ay = c.by = c.cy = c.dy = c.az = c.bz = c.cz = c.dz = 0.0;
        return c;
    }
    double c1 = 6.0 * P / (5.0 * L), c2 = P / 10.0, c3 = 2.0 * P * L / 15.0, c4 = -P * L / 30.0;
    c.ay = c.az = c1; c.by = c.bz = c2; c.cy = c.cz = c3; c.dy = c.dz = c4;
    return c;
}

// out = k^{xy}_{AB} M: the 3x3 local sub-block (node A part x, node B part
// y; part 0 = translations, 1 = rotations) times a 3x3 matrix.
template <int A, int B, int X, int Y>
__device__ __forceinline__ void kmul(const FrameK &c, const double *M, double out[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
#pragma unroll
            for (int l = 0; l < 3; ++l)
                if (frame_nz(6 * A + 3 * X + i, 6 * B + 3 * Y + l))
                    s += frame_k(c, 6 * A + 3 * X + i, 6 * B + 3 * Y + l) * M[3 * l + j];
            out[i][j] = s;
        }
}

// acc (+)= P^T W for a 3x3 P (row-major) and W.
__device__ __forceinline__ void tmul(const double *P, const double W[3][3], double acc[3][3], bool add) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = P[i] * W[0][j] + P[3 + i] * W[1][j] + P[6 + i] * W[2][j];
            acc[i][j] = add ? acc[i][j] + s : s;
        }
}

// sb: the thread's staged slot in shared memory in stored orientation, or
// null to write through blk_entry.  K: the 36 values row-major.  KG: the
// translation 3x3 and its padding (12), then the rotation sub-blocks as
// blk_entry places them in kg_rot (kKgRotStride).
__device__ __forceinline__ void bar_store(const ElemOut &o, int64_t e, int32_t sl, int bi, int bj, const double G[3][3],
                                          bool diag, int node, double &lmax, int64_t pair_id, double *sb) {
    const bool t = sl & kBlkTranspose;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            lmax = fmax(lmax, fabs(G[i][j]));
            const int r0 = 3 * bi + i, c0 = 3 * bj + j;
            if (sb) {
                const int r = t ? c0 : r0, c = t ? r0 : c0;
                if (!o.kg_layout) sb[6 * r + c] = G[i][j];
                else if (r < 3 && c < 3) sb[3 * r + c] = G[i][j];
                else sb[12 + 9 * (2 * (r / 3) + c / 3 - 1) + 3 * (r % 3) + (c % 3)] = G[i][j];
            } else {
                *blk_entry(o, sl, r0, c0, pair_id) = G[i][j];
            }
        }
    if (diag && o.diag_staging && bi == bj)
#pragma unroll
        for (int i = 0; i < 3; ++i) o.diag_staging[__ldg(o.diag_slot + e * 12 + 6 * node + 3 * bi + i)] = G[i][i];
}

// Global node-pair block (A, B) of T' k T with T_n = [[R_n, O_n], [0, R_n]]
// (R_n = Rel node_R_n, O_n = -Rel skew(w_n) node_R_n):
//   G_tt = R_A' k_tt R_B               G_tr = R_A' (k_tt O_B + k_tr R_B)
//   G_rt = O_A' k_tt R_B + R_A' k_rt R_B
//   G_rr = O_A' (k_tt O_B + k_tr R_B) + R_A' (k_rt O_B + k_rr R_B)
// With a shared buffer sbuf, a regular slot is staged there and sent out as
// bulk copies (K: one of 288 bytes; KG: the translation slot, 96 bytes, and the
// rotation record, 224); RBE2-path slots are written directly.
template <int A, int B>
__device__ __forceinline__ void bar_pair(const ElemOut &o, int64_t e, int p, const BarFrame &F, const FrameK &c,
                                         double &lmax, double *sbuf = nullptr) {
    const int32_t sl = __ldg(o.blk_slot + e * 3 + p);
    double *sb = sl >= 0 ? sbuf : nullptr;
    const bool off = F.off;
    const double *RA = F.TR[A], *RB = F.TR[B], *OA = F.Toff[A], *OB = F.Toff[B];
    double W[3][3], W2[3][3], G[3][3];
    // tt
    kmul<A, B, 0, 0>(c, RB, W);
    tmul(RA, W, G, false);
    bar_store(o, e, sl, 0, 0, G, A == B, A, lmax, 3 * e + p, sb);
    // rt (W = k_tt R_B)
    kmul<A, B, 1, 0>(c, RB, W2);
    tmul(RA, W2, G, false);
    if (off) tmul(OA, W, G, true);
    bar_store(o, e, sl, 1, 0, G, false, A, lmax, 3 * e + p, sb);
    // tr: W = k_tt O_B + k_tr R_B
    kmul<A, B, 0, 1>(c, RB, W);
    if (off) {
        kmul<A, B, 0, 0>(c, OB, W2);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) W[i][j] = W2[i][j] + W[i][j];
    }
    tmul(RA, W, G, false);
    bar_store(o, e, sl, 0, 1, G, false, A, lmax, 3 * e + p, sb);
    // rr: R_A' (k_rt O_B + k_rr R_B) + O_A' W
    kmul<A, B, 1, 1>(c, RB, W2);
    if (off) {
        double W3[3][3];
        kmul<A, B, 1, 0>(c, OB, W3);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) W2[i][j] = W3[i][j] + W2[i][j];
    }
    tmul(RA, W2, G, false);
    if (off) tmul(OA, W, G, true);
    bar_store(o, e, sl, 1, 1, G, A == B, A, lmax, 3 * e + p, sb);
    if (sb) {
        const int64_t idx = sl & kBlkIndexMask;
        if (!o.kg_layout) {
            slot_fence();
            slot_copy(o.staging + 36 * idx, sb, 288);
        } else {
            sb[9] = 0.0; sb[10] = 0.0; sb[11] = 0.0; sb[12 + 27] = 0.0;  // padding
            slot_fence();
            slot_copy(o.staging + 12 * idx, sb, 96);
            slot_copy(o.kg_rot + kKgRotStride * (3 * e + p), sb + 12, 8 * kKgRotStride);
        }
    }
}

// One (bar, node pair) per thread, pair-major so that a warp runs one
// compile-time pair; each of the three threads recomputes the bar frame.
// Dynamic shared memory: kBarSlotStride doubles per thread, the staged slot.
constexpr int kBarSlotStride = 38;  // 16-byte aligned, and off the 36-double bank period
constexpr int kBarKgSlotStride = 42;  // KG: 12 + kKgRotStride values, 16-byte aligned
__global__ void __launch_bounds__(128, 3) bar_k_kernel(int64_t nb, const int32_t *__restrict__ nodes,
                                                      const double *__restrict__ prop, const double *__restrict__ coords,
                                                      const double *__restrict__ nodeR, ElemOut o) {
    extern __shared__ __align__(16) double bar_smem[];
    double *sbuf = bar_smem + kBarSlotStride * threadIdx.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int pair = (int)(t / nb);
    const int64_t e = t - (int64_t)pair * nb;
    o = o.at(blockIdx.y);
    if (o.bprop) prop = o.bprop;
    double lmax = 0.0;
    if (pair < 3) {
        BarFrame F;
        int32_t nd[2];
        if (bar_frame(e, nodes, prop, coords, nodeR, F, nd)) {
            const FrameK c = frame3d_k(prop + 18 * e, F.L);
            if (pair == 0) bar_pair<0, 0>(o, e, 0, F, c, lmax, sbuf);
            else if (pair == 1) bar_pair<0, 1>(o, e, 1, F, c, lmax, sbuf);
            else bar_pair<1, 1>(o, e, 2, F, c, lmax, sbuf);
        }
    }
    if (o.maxabs) {
        for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
        if ((threadIdx.x & 31) == 0 && lmax > 0.0) atomic_max_nonneg(o.maxabs, lmax);
    }
    slot_copies_read();
}

// Dynamic shared memory: kBarKgSlotStride doubles per thread, the staged slot.
__global__ void __launch_bounds__(128, 3) bar_kg_kernel(int64_t nb, const int32_t *__restrict__ nodes,
                                                       const double *__restrict__ prop, const double *__restrict__ coords,
                                                       const double *__restrict__ nodeR, const double *__restrict__ u,
                                                       ElemOut o) {
    extern __shared__ __align__(16) double bar_kg_smem[];
    double *sbuf = bar_kg_smem + kBarKgSlotStride * threadIdx.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int pair = (int)(t / nb);
    const int64_t e = t - (int64_t)pair * nb;
    if (pair >= 3) return;
    o = o.at(blockIdx.y);
    if (o.bprop) prop = o.bprop;
    u += (int64_t)blockIdx.y * o.u_stride;
    BarFrame F;
    int32_t nd[2];
    if (!bar_frame(e, nodes, prop, coords, nodeR, F, nd)) return;
    // axial force P = (k u_bar)[7] (forces_frame3d): row 7 of k has only the
    // axial entries, and u_bar's axial components are (R_n u_n + O_n theta_n)_x.
    double ux[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double *ug = u + 6 * (int64_t)nd[k];
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 3; ++q) s += F.TR[k][q] * __ldg(ug + q);
#pragma unroll
        for (int q = 0; q < 3; ++q) s += F.Toff[k][q] * __ldg(ug + 3 + q);
        ux[k] = s;
    }
    const double *pr = prop + 18 * e;
    double A = __ldg(pr), E = __ldg(pr + 7);
    double X = E * A / F.L;
    double P = -X * ux[0] + X * ux[1];
    const FrameK c = frame3d_kg(F.L, P);
    double lmax = 0.0;
    if (pair == 0) bar_pair<0, 0>(o, e, 0, F, c, lmax, sbuf);
    else if (pair == 1) bar_pair<0, 1>(o, e, 1, F, c, lmax, sbuf);
    else bar_pair<1, 1>(o, e, 2, F, c, lmax, sbuf);
    slot_copies_read();
}

}  // namespace jfg
