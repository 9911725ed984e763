// elem_q4.cuh -- CQUAD4 stiffness (K) and differential stiffness (KG) kernels.
//
// Mapping: a team of 10 lanes owns one element, three teams per warp
// (lanes 30-31 only join the warp barriers).  Per-element intermediates live
// in shared memory; the final phase gives each lane one node pair (a <= b)
// of the symmetric 24x24 global matrix, so the 300 packed values are
// produced without redundant work and written straight to their sorted
// contribution slots (deterministic segmented reduction follows).
//
// K follows stiffness_quad4_matrices' default planar branch
// (src/FEMKernels.jl:3185-4034): 2x2 Gauss membrane + bending with the
// MacNeal twist row (:3670-3673), Hughes-Brezzi drilling (:3556-3559,
// :3778-3779), Wilson incompatible modes condensed by 4x4 inverses
// (:3790-3801, :3964-4011) and MacNeal's residual-bending-flexibility shear
// (add_quad4_macneal_shear_rbf!, :4715-4978); then T'KT with T built from the
// element frame and node CD frames (src/solver/assembly.jl:3808-3837).
//
// KG follows the Q4 branch of the shell loop of assemble_geometric_stiffness
// (assembly.jl:4812-6017): u_elem = T u (:5176-5185), membrane resultants with
// incompatible modes (quad4_membrane_force_field, FEMKernels.jl:6341-6539),
// Gauss-point stresses N/h (:5475-5541), geometric_stiffness_quad4 with the
// principal-transverse operator and the incompatible-mode condensation map
// (FEMKernels.jl:7554-7985, :6708-6785, :6891-6972), T'KgT and the drill
// zeroing (:5978-6007).  The principal-transverse term per Gauss point and
// principal direction (c, s) is the rank-one form
//   f * [(s*gx - c*gy)(s*gx - c*gy)' + gz gz'],  f = h |J| lambda,
// which is the reference's p11/p22/p12 expansion factored.
#pragma once
#include "jfg_common.cuh"

namespace jfg {

constexpr int Q4_TEAM = 10;
constexpr int Q4_TEAMS_PER_WARP = 3;
constexpr int Q4_WARPS = 4;
constexpr int Q4_THREADS = 32 * Q4_WARPS;
constexpr int Q4_ELEMS_PER_BLOCK = Q4_TEAMS_PER_WARP * Q4_WARPS;
constexpr int Q4_PACKED = 300;

__constant__ int c_pair_a[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
__constant__ int c_pair_b[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};

// Output of an element kernel.  Every element node pair (a <= b) owns one
// 36-double block: rows = dofs of local node a, columns = dofs of node b.
//   blk_slot >= 0: block index in `staging` (bits 0..29) with bit 30 set when
//                  the global node order is reversed (the block is stored
//                  transposed so that it reads as rows of the lower-numbered
//                  node);
//   blk_slot <  0: the pair touches an RBE2 node; the raw block goes to
//                  exc_raw[36 * (-slot - 1)] for the dof-level expansion.
//
// Batched variants: a launch may cover several variants of one model
// (blockIdx.y = variant).  They share the mesh, the pattern and the maps;
// each has its own staging, raw RBE2 blocks, diagonal staging and max, its
// own displacement field, and optionally its own shell thicknesses and bar
// records.  A single-model call is the one-variant case with zero strides.
struct ElemOut {
    double *staging = nullptr;           // 36 doubles per sorted block slot
    double *exc_raw = nullptr;           // 36 doubles per constraint-touching pair
    const int32_t *blk_slot = nullptr;   // per element node pair
    double *diag_staging = nullptr;      // K only: raw element diagonal at sorted dof slots (or null)
    const int32_t *diag_slot = nullptr;  // per element local dof (or null)
    double *maxabs = nullptr;            // K only: max |value| (bit-pattern atomic), or null
    int64_t staging_stride = 0, exc_stride = 0, dstage_stride = 0;  // per-variant output strides
    const double *h = nullptr;           // per-variant shell thickness of this element type, or null
    int64_t h_stride = 0;
    const double *bprop = nullptr;       // per-variant bar records, or null
    int64_t bprop_stride = 0;
    int64_t u_stride = 0;                // per-variant displacement stride (ndof)

    __device__ __forceinline__ ElemOut at(int v) const {
        ElemOut r = *this;
        r.staging += v * staging_stride;
        r.exc_raw += v * exc_stride;
        if (diag_staging) r.diag_staging += v * dstage_stride;
        if (maxabs) r.maxabs += v;
        if (h) r.h += v * h_stride;
        if (bprop) r.bprop += v * bprop_stride;
        return r;
    }
    // Shell thickness of element e: the variant's own, else the property record's.
    __device__ __forceinline__ double thickness(int64_t e, const double *pr) const { return h ? __ldg(h + e) : __ldg(pr); }
};

constexpr int32_t kBlkTranspose = 1 << 30;
constexpr int32_t kBlkIndexMask = kBlkTranspose - 1;

// Address of entry (i, j) of a pair block given its slot.
__device__ __forceinline__ double *blk_entry(const ElemOut &o, int32_t s, int i, int j) {
    if (s < 0) return o.exc_raw + 36 * (int64_t)(-(s + 1)) + 6 * i + j;
    double *base = o.staging + 36 * (int64_t)(s & kBlkIndexMask);
    return (s & kBlkTranspose) ? base + 6 * j + i : base + 6 * i + j;
}

struct Q4Geo {
    double p[4][3];
    double v[3][3];
    double lc[4][2];
    double Q[4][9];
    double dNx[5][4], dNy[5][4];  // 4 Gauss points + centre (index 4)
    double wdet[4];
    double dphi[4][4];            // d1x, d1y, d2x, d2y per Gauss point
};

struct Q4KShared {
    Q4Geo g;
    double Cm[9], Cb[9], Cs[4];
    double h, alpha_d;
    int skip_macneal, bend_cond;
    double Kabm[8][4], Kbbm[16], Kabb[8][4], Kbbb[16];
    double D[4][12], Jp[4];
    MacNealZ mz;
    union {
        double P[2][4][4][3];  // phase 1: C b_l(g) for membrane (0) / bending (1) incompatible modes
        struct {
            double Xm[4][8], Xb[4][8];
            double Y[4][12];
        } x;                   // phases 3-4
    } u;
};

struct Q4GShared {
    Q4Geo g;
    double Cm[9], h;
    double uuv[8];
    double P[4][4][3];  // Cm b_l(g) of the membrane incompatible modes
    double Kabm[8][4], Kbbm[16];
    double Am[4][8];
    double alpha[4];
    double t[8][8], gz[8][4], f[8];
};

__device__ __forceinline__ void q4_shape_gp(int g, double &r, double &s) {
    const double pt = 0.57735026918962576451;  // 1/sqrt(3)
    r = (g == 0 || g == 3) ? -pt : pt;
    s = (g <= 1) ? -pt : pt;
}

__device__ __forceinline__ double q4_N(int k, double r, double s) {
    return 0.25 * (1 + ((k == 1 || k == 2) ? r : -r)) * (1 + (k >= 2 ? s : -s));
}

// Phase 0 of both kernels: node loads, frame, local coordinates, node
// transformation blocks and Gauss-point Jacobians.  Called by all lanes of
// a team; `tl` is the lane index within the team, `valid` false for teams
// past the end (they still reach every barrier).
__device__ __forceinline__ void q4_geometry(Q4Geo &G, int tl, bool valid, const int32_t *nd,
                                            const double *__restrict__ coords, const double *__restrict__ nodeR) {
    if (valid && tl < 4) {
        int n = nd[tl];
        G.p[tl][0] = __ldg(coords + 3 * (int64_t)n);
        G.p[tl][1] = __ldg(coords + 3 * (int64_t)n + 1);
        G.p[tl][2] = __ldg(coords + 3 * (int64_t)n + 2);
    }
    __syncwarp();
    if (valid && tl == 0) {
        double v1[3], v2[3], v3[3];
        q4_frame(G.p[0], G.p[1], G.p[2], G.p[3], v1, v2, v3);
        double c[3];
        for (int i = 0; i < 3; ++i) c[i] = (G.p[0][i] + G.p[1][i] + G.p[2][i] + G.p[3][i]) / 4.0;
        for (int k = 0; k < 4; ++k) {
            double d[3];
            sub3(G.p[k], c, d);
            G.lc[k][0] = dot3(d, v1);
            G.lc[k][1] = dot3(d, v2);
        }
        for (int i = 0; i < 3; ++i) { G.v[0][i] = v1[i]; G.v[1][i] = v2[i]; G.v[2][i] = v3[i]; }
    }
    __syncwarp();
    if (valid && tl < 4) {
        const double *R = nodeR ? nodeR + 9 * (int64_t)nd[tl] : nullptr;
        double Rl[9];
        if (R)
            for (int i = 0; i < 9; ++i) Rl[i] = __ldg(R + i);
        node_block(G.v[0], G.v[1], G.v[2], R ? Rl : nullptr, G.Q[tl]);
    } else if (valid && tl < 9) {
        int g = tl - 4;  // 0..3 Gauss points, 4 = centre
        double r = 0.0, s = 0.0;
        if (g < 4) q4_shape_gp(g, r, s);
        double dNr[4] = {-0.25 * (1 - s), 0.25 * (1 - s), 0.25 * (1 + s), -0.25 * (1 + s)};
        double dNs[4] = {-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r), 0.25 * (1 - r)};
        double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
        for (int k = 0; k < 4; ++k) {
            J11 += dNr[k] * G.lc[k][0]; J12 += dNr[k] * G.lc[k][1];
            J21 += dNs[k] * G.lc[k][0]; J22 += dNs[k] * G.lc[k][1];
        }
        double det = J11 * J22 - J12 * J21;
        double inv = 1.0 / det;
        double iJ11 = J22 * inv, iJ12 = -J12 * inv, iJ21 = -J21 * inv, iJ22 = J11 * inv;
        for (int k = 0; k < 4; ++k) {
            G.dNx[g][k] = iJ11 * dNr[k] + iJ12 * dNs[k];
            G.dNy[g][k] = iJ21 * dNr[k] + iJ22 * dNs[k];
        }
        if (g < 4) {
            double a = fabs(det);
            G.wdet[g] = a < 1e-12 ? 1e-12 : a;
            G.dphi[g][0] = iJ11 * (-2.0 * r);
            G.dphi[g][1] = iJ21 * (-2.0 * r);
            G.dphi[g][2] = iJ12 * (-2.0 * s);
            G.dphi[g][3] = iJ22 * (-2.0 * s);
        }
    }
}

// Bending B column of local dof (theta_x: comp 0, theta_y: comp 1) of node k
// at Gauss point g, with the MacNeal twist correction.
__device__ __forceinline__ void q4_bend_col(const Q4Geo &G, int g, int k, int comp, double b[3]) {
    double x = G.dNx[g][k], y = G.dNy[g][k];
    if (comp == 0) { b[0] = 0.0; b[1] = -y; b[2] = 2.0 * (-x) - (-G.dNx[4][k]); }
    else { b[0] = x; b[1] = 0.0; b[2] = 2.0 * y - G.dNy[4][k]; }
}
__device__ __forceinline__ void q4_mem_col(const Q4Geo &G, int g, int k, int comp, double b[3]) {
    double x = G.dNx[g][k], y = G.dNy[g][k];
    if (comp == 0) { b[0] = x; b[1] = 0.0; b[2] = y; }
    else { b[0] = 0.0; b[1] = y; b[2] = x; }
}
// Membrane incompatible-mode column l (0..3) at Gauss point g.
__device__ __forceinline__ void q4_bi_col(const Q4Geo &G, int g, int l, double b[3]) {
    double d1x = G.dphi[g][0], d1y = G.dphi[g][1], d2x = G.dphi[g][2], d2y = G.dphi[g][3];
    switch (l) {
        case 0: b[0] = d1x; b[1] = 0.0; b[2] = d1y; break;
        case 1: b[0] = 0.0; b[1] = d1y; b[2] = d1x; break;
        case 2: b[0] = d2x; b[1] = 0.0; b[2] = d2y; break;
        default: b[0] = 0.0; b[1] = d2y; b[2] = d2x; break;
    }
}
// Bending incompatible-mode column l (0..3) at Gauss point g.
__device__ __forceinline__ void q4_bib_col(const Q4Geo &G, int g, int l, double b[3]) {
    double d1x = G.dphi[g][0], d1y = G.dphi[g][1], d2x = G.dphi[g][2], d2y = G.dphi[g][3];
    switch (l) {
        case 0: b[0] = 0.0; b[1] = -d1y; b[2] = -d1x; break;
        case 1: b[0] = 0.0; b[1] = -d2y; b[2] = -d2x; break;
        case 2: b[0] = d1x; b[1] = 0.0; b[2] = d1y; break;
        default: b[0] = d2x; b[1] = 0.0; b[2] = d2y; break;
    }
}
__device__ __forceinline__ double quad_form(const double a[3], const double C[9], const double b[3]) {
    double cb0 = C[0] * b[0] + C[1] * b[1] + C[2] * b[2];
    double cb1 = C[3] * b[0] + C[4] * b[1] + C[5] * b[2];
    double cb2 = C[6] * b[0] + C[7] * b[1] + C[8] * b[2];
    return a[0] * cb0 + a[1] * cb1 + a[2] * cb2;
}

// G = Qa^T L Qb for one 3x3 sub-block.
__device__ __forceinline__ void rot_block(const double *Qa, const double L[3][3], const double *Qb, double out[3][3]) {
    double W[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) W[i][j] = L[i][0] * Qb[j] + L[i][1] * Qb[3 + j] + L[i][2] * Qb[6 + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[i][j] = Qa[i] * W[0][j] + Qa[3 + i] * W[1][j] + Qa[6 + i] * W[2][j];
}

// Write one global 6x6 node-pair block (a <= b, pair index p) of element e
// with NP node pairs; diagonal entries of diagonal pairs also go to the
// orig_diag staging (K only).
template <int NN, int NP>
__device__ __forceinline__ void write_pair_block(const ElemOut &o, int64_t e, int p, int a, int b, const double Gb[6][6],
                                                 double &lmax) {
    const int32_t s = __ldg(o.blk_slot + e * NP + p);
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            double v = Gb[i][j];
            lmax = fmax(lmax, fabs(v));
            *blk_entry(o, s, i, j) = v;
        }
    if (o.diag_staging && a == b) {
#pragma unroll
        for (int i = 0; i < 6; ++i) o.diag_staging[__ldg(o.diag_slot + e * 6 * NN + 6 * a + i)] = Gb[i][i];
    }
}

// Write one 3x3 sub-block (bi, bj) of the node-pair block (a, b) of element
// e; diagonal entries of diagonal pairs also go to the orig_diag staging.
__device__ __forceinline__ void write_sub_block(const ElemOut &o, int64_t e, int32_t sl, int a, int b, int bi, int bj,
                                                const double O[3][3], double &lmax, int ndof_e) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double v = O[i][j];
            lmax = fmax(lmax, fabs(v));
            *blk_entry(o, sl, 3 * bi + i, 3 * bj + j) = v;
        }
    if (o.diag_staging && a == b && bi == bj) {
#pragma unroll
        for (int i = 0; i < 3; ++i) o.diag_staging[__ldg(o.diag_slot + e * ndof_e + 6 * a + 3 * bi + i)] = O[i][i];
    }
}

__global__ void __launch_bounds__(Q4_THREADS, 4) q4_k_kernel(int64_t nq, const int32_t *__restrict__ nodes,
                                                         const double *__restrict__ prop,
                                                         const double *__restrict__ coords,
                                                         const double *__restrict__ nodeR, double k6rot, ElemOut o) {
    __shared__ Q4KShared sh[Q4_ELEMS_PER_BLOCK];
    o = o.at(blockIdx.y);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane / Q4_TEAM, tl = lane - team * Q4_TEAM;
    const bool in_team = team < Q4_TEAMS_PER_WARP;
    const int slot_id = warp * Q4_TEAMS_PER_WARP + (in_team ? team : 0);
    const int64_t e = (int64_t)blockIdx.x * Q4_ELEMS_PER_BLOCK + slot_id;
    const bool valid = in_team && e < nq;
    Q4KShared &S = sh[slot_id];
    int32_t nd[4] = {0, 0, 0, 0};
    // property loads are issued before the geometry so that their latency
    // overlaps the node and coordinate loads
    double h = 0.0, E = 0.0, nu = 0.0, br = 0.0, tst = 0.0, Gs = 0.0;
    if (valid && tl == 9) {
        const double *pr = prop + 7 * e;
        h = o.thickness(e, pr); E = __ldg(pr + 1); nu = __ldg(pr + 2); br = __ldg(pr + 4); tst = __ldg(pr + 5);
        Gs = __ldg(pr + 6);
    }
    if (valid)
        for (int k = 0; k < 4; ++k) nd[k] = __ldg(nodes + 4 * e + k);

    q4_geometry(S.g, in_team ? tl : 99, valid, nd, coords, nodeR);
    if (valid && tl == 9) {
        // constitutive build for isotropic PSHELL/MAT1 (assembly.jl:2460-2469)
        double cm = E * h / (1 - nu * nu);
        double cb = br * (E * h * h * h) / (12 * (1 - nu * nu));
        double base[9] = {1.0, nu, 0.0, nu, 1.0, 0.0, 0.0, 0.0, (1 - nu) / 2};
        for (int i = 0; i < 9; ++i) { S.Cm[i] = cm * base[i]; S.Cb[i] = cb * base[i]; }
        bool membrane_only = br <= 1e-12;
        double cs = membrane_only ? 0.0 : tst * h * Gs;
        S.Cs[0] = cs; S.Cs[1] = 0.0; S.Cs[2] = 0.0; S.Cs[3] = cs;
        S.h = h;
        double G_drill = S.Cm[8] / h;
        if (G_drill < 1e-6) G_drill = E / (2 * 3.0);
        double k6 = membrane_only ? 0.0 : k6rot, ds = membrane_only ? 0.0 : 1.0;
        S.alpha_d = ds * (k6 / 1e5) * G_drill * h;
        S.skip_macneal = (h < 1e-30 || fabs(cs) < 1e-30) ? 1 : 0;
    }
    __syncwarp();

    // Phase 1: MacNeal strain-sampling rows, incompatible-mode couplings.
    if (valid && tl < 4) {
        const double pt = 0.57735026918962576451;
        const double xs[4] = {0.0, 0.0, -pt, pt}, es[4] = {-pt, pt, 0.0, 0.0};
        double xi = xs[tl], eta = es[tl];
        double dNr[4] = {-0.25 * (1 - eta), 0.25 * (1 - eta), 0.25 * (1 + eta), -0.25 * (1 + eta)};
        double dNs[4] = {-0.25 * (1 - xi), -0.25 * (1 + xi), 0.25 * (1 + xi), 0.25 * (1 - xi)};
        double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
        for (int k = 0; k < 4; ++k) {
            J11 += dNr[k] * S.g.lc[k][0]; J12 += dNr[k] * S.g.lc[k][1];
            J21 += dNs[k] * S.g.lc[k][0]; J22 += dNs[k] * S.g.lc[k][1];
        }
        double det = J11 * J22 - J12 * J21;
        if (fabs(det) < 1e-14) det = det < 0.0 ? -1e-14 : 1e-14;
        S.Jp[tl] = fabs(det);
        double inv = 1.0 / det;
        double iJ11 = J22 * inv, iJ12 = -J12 * inv, iJ21 = -J21 * inv, iJ22 = J11 * inv;
        for (int k = 0; k < 4; ++k) {
            double dx = iJ11 * dNr[k] + iJ12 * dNs[k];
            double dy = iJ21 * dNr[k] + iJ22 * dNs[k];
            double Nk = 0.25 * (1 + ((k == 1 || k == 2) ? xi : -xi)) * (1 + (k >= 2 ? eta : -eta));
            if (tl < 2) { S.D[tl][3 * k] = dx; S.D[tl][3 * k + 1] = 0.0; S.D[tl][3 * k + 2] = Nk; }
            else { S.D[tl][3 * k] = dy; S.D[tl][3 * k + 1] = -Nk; S.D[tl][3 * k + 2] = 0.0; }
        }
    }
    // C b_l(g) of every incompatible-mode column (membrane, bending).
    if (valid) {
        for (int w = tl; w < 32; w += Q4_TEAM) {
            const int kind = w >> 4, g = (w >> 2) & 3, l = w & 3;
            double b[3];
            if (kind == 0) q4_bi_col(S.g, g, l, b);
            else q4_bib_col(S.g, g, l, b);
            const double *C = kind == 0 ? S.Cm : S.Cb;
#pragma unroll
            for (int r = 0; r < 3; ++r) S.u.P[kind][g][l][r] = C[3 * r] * b[0] + C[3 * r + 1] * b[1] + C[3 * r + 2] * b[2];
        }
    }
    __syncwarp();
    // K_ab / K_bb rows (membrane then bending): 8 + 4 + 8 + 4 row items,
    // four independent accumulators each.
    if (valid) {
        for (int w = tl; w < 24; w += Q4_TEAM) {
            const int kind = w >= 12 ? 1 : 0, r = w - 12 * kind;
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                double a[3];
                if (r < 8) {
                    if (kind == 0) q4_mem_col(S.g, g, r >> 1, r & 1, a);
                    else q4_bend_col(S.g, g, r >> 1, r & 1, a);
                } else {
                    if (kind == 0) q4_bi_col(S.g, g, r - 8, a);
                    else q4_bib_col(S.g, g, r - 8, a);
                }
                const double wd = S.g.wdet[g];
#pragma unroll
                for (int l = 0; l < 4; ++l) {
                    const double *P = S.u.P[kind][g][l];
                    acc[l] += wd * (a[0] * P[0] + a[1] * P[1] + a[2] * P[2]);
                }
            }
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                if (r < 8) (kind == 0 ? S.Kabm : S.Kabb)[r][l] = acc[l];
                else (kind == 0 ? S.Kbbm : S.Kbbb)[4 * (r - 8) + l] = acc[l];
            }
        }
    }
    __syncwarp();

    // Phase 2: the two 4x4 inverses (lanes 0 and 1 in one code path) and the
    // MacNeal compliance factors (lane 2).
    if (valid && tl < 2) {
        double *M = tl == 0 ? S.Kbbm : S.Kbbb;
        bool inv = true;
        if (tl == 1) {
            double mx = 0.0;
            for (int i = 0; i < 16; ++i) mx = fmax(mx, fabs(M[i]));
            S.bend_cond = mx > 0.0 ? 1 : 0;
            inv = mx > 0.0;
        }
        if (inv) inv4_inplace(M);
    } else if (valid && tl == 2 && !S.skip_macneal) {
        S.mz = macneal_z(S.g.lc, S.Jp, S.Cs[0], S.Cb[0], S.Cb[4]);
    }
    __syncwarp();

    // Phase 3: X = Kbb^-1 Kab' for both condensations, Y = Z \ D by columns.
    if (valid) {
        for (int w = tl; w < 76; w += Q4_TEAM) {
            if (w < 32) {
                int l = w >> 3, r = w & 7;
                double s = 0.0;
                for (int q = 0; q < 4; ++q) s += S.Kbbm[4 * l + q] * S.Kabm[r][q];
                S.u.x.Xm[l][r] = s;
            } else if (w < 64) {
                int l = (w - 32) >> 3, r = (w - 32) & 7;
                double s = 0.0;
                if (S.bend_cond)
                    for (int q = 0; q < 4; ++q) s += S.Kbbb[4 * l + q] * S.Kabb[r][q];
                S.u.x.Xb[l][r] = s;
            } else if (!S.skip_macneal) {
                int j = w - 64;
                double d[4] = {S.D[0][j], S.D[1][j], S.D[2][j], S.D[3][j]}, y[4];
                macneal_y(S.mz, d, y);
                for (int l = 0; l < 4; ++l) S.u.x.Y[l][j] = y[l];
            }
        }
    }
    __syncwarp();

    // Phase 4: one node pair per lane.
    double lmax = 0.0;
    if (valid) {
        const int a = c_pair_a[tl], b = c_pair_b[tl];
        double L[6][6];
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = 0; j < 6; ++j) L[i][j] = 0.0;
        const double ad = S.alpha_d;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            double r, s;
            q4_shape_gp(g, r, s);
            const double wd = S.g.wdet[g];
            double ma[2][3], mb[2][3], ba[2][3], bb[2][3];
            q4_mem_col(S.g, g, a, 0, ma[0]); q4_mem_col(S.g, g, a, 1, ma[1]);
            q4_mem_col(S.g, g, b, 0, mb[0]); q4_mem_col(S.g, g, b, 1, mb[1]);
            q4_bend_col(S.g, g, a, 0, ba[0]); q4_bend_col(S.g, g, a, 1, ba[1]);
            q4_bend_col(S.g, g, b, 0, bb[0]); q4_bend_col(S.g, g, b, 1, bb[1]);
#pragma unroll
            for (int be = 0; be < 2; ++be) {
                double cm[3], cb[3];
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    cm[r] = wd * (S.Cm[3 * r] * mb[be][0] + S.Cm[3 * r + 1] * mb[be][1] + S.Cm[3 * r + 2] * mb[be][2]);
                    cb[r] = wd * (S.Cb[3 * r] * bb[be][0] + S.Cb[3 * r + 1] * bb[be][1] + S.Cb[3 * r + 2] * bb[be][2]);
                }
#pragma unroll
                for (int al = 0; al < 2; ++al) {
                    L[al][be] += ma[al][0] * cm[0] + ma[al][1] * cm[1] + ma[al][2] * cm[2];
                    L[3 + al][3 + be] += ba[al][0] * cb[0] + ba[al][1] * cb[1] + ba[al][2] * cb[2];
                }
            }
            // drilling: Bd = [0.5 dN/dy, -0.5 dN/dx, N] on (u, v, theta_z)
            double da[3] = {0.5 * S.g.dNy[g][a], -0.5 * S.g.dNx[g][a], q4_N(a, r, s)};
            double db[3] = {0.5 * S.g.dNy[g][b], -0.5 * S.g.dNx[g][b], q4_N(b, r, s)};
            const int di[3] = {0, 1, 5};
            double wda = wd * ad;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) L[di[i]][di[j]] += wda * da[i] * db[j];
        }
        if (!S.skip_macneal) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int l = 0; l < 4; ++l) {
                        s1 += S.D[l][3 * a + i] * S.u.x.Y[l][3 * b + j];
                        s2 += S.D[l][3 * b + j] * S.u.x.Y[l][3 * a + i];
                    }
                    L[2 + i][2 + j] += 0.5 * (s1 + s2);
                }
        }
#pragma unroll
        for (int al = 0; al < 2; ++al)
#pragma unroll
            for (int be = 0; be < 2; ++be) {
                double sm = 0.0, sb = 0.0;
                for (int l = 0; l < 4; ++l) {
                    sm += S.Kabm[2 * a + al][l] * S.u.x.Xm[l][2 * b + be];
                    sb += S.Kabb[2 * a + al][l] * S.u.x.Xb[l][2 * b + be];
                }
                L[al][be] -= sm;
                if (S.bend_cond) L[3 + al][3 + be] -= sb;
            }
        // T'KT on the node pair, one 3x3 sub-block at a time (keeps the
        // register footprint to the local 6x6 block)
        const int32_t sl = __ldg(o.blk_slot + e * 10 + tl);
#pragma unroll
        for (int bi = 0; bi < 2; ++bi)
#pragma unroll
            for (int bj = 0; bj < 2; ++bj) {
                double Ls[3][3], O[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) Ls[i][j] = L[3 * bi + i][3 * bj + j];
                rot_block(S.g.Q[a], Ls, S.g.Q[b], O);
                write_sub_block(o, e, sl, a, b, bi, bj, O, lmax, 24);
            }
    }
    if (o.maxabs) {
        for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
        if (lane == 0 && lmax > 0.0) atomic_max_nonneg(o.maxabs, lmax);
    }
}

__global__ void __launch_bounds__(Q4_THREADS) q4_kg_kernel(int64_t nq, const int32_t *__restrict__ nodes,
                                                          const double *__restrict__ prop,
                                                          const double *__restrict__ coords,
                                                          const double *__restrict__ nodeR,
                                                          const double *__restrict__ u, ElemOut o) {
    __shared__ Q4GShared sh[Q4_ELEMS_PER_BLOCK];
    o = o.at(blockIdx.y);
    u += (int64_t)blockIdx.y * o.u_stride;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane / Q4_TEAM, tl = lane - team * Q4_TEAM;
    const bool in_team = team < Q4_TEAMS_PER_WARP;
    const int slot_id = warp * Q4_TEAMS_PER_WARP + (in_team ? team : 0);
    const int64_t e = (int64_t)blockIdx.x * Q4_ELEMS_PER_BLOCK + slot_id;
    const bool valid = in_team && e < nq;
    Q4GShared &S = sh[slot_id];
    int32_t nd[4] = {0, 0, 0, 0};
    if (valid)
        for (int k = 0; k < 4; ++k) nd[k] = __ldg(nodes + 4 * e + k);

    q4_geometry(S.g, in_team ? tl : 99, valid, nd, coords, nodeR);
    if (valid && tl == 9) {
        const double *pr = prop + 7 * e;
        double h = o.thickness(e, pr), E = __ldg(pr + 1), nu = __ldg(pr + 2);
        double cm = E / (1 - nu * nu);
        double base[9] = {1.0, nu, 0.0, nu, 1.0, 0.0, 0.0, 0.0, (1 - nu) / 2};
        for (int i = 0; i < 9; ++i) S.Cm[i] = (cm * base[i]) * h;
        S.h = h;
    }
    __syncwarp();
    // local membrane displacements u_elem = T u_global (u, v of each node)
    if (valid && tl < 4) {
        const double *ug = u + 6 * (int64_t)nd[tl];
        double u0 = __ldg(ug), u1 = __ldg(ug + 1), u2 = __ldg(ug + 2);
        const double *Q = S.g.Q[tl];
        S.uuv[2 * tl] = Q[0] * u0 + Q[1] * u1 + Q[2] * u2;
        S.uuv[2 * tl + 1] = Q[3] * u0 + Q[4] * u1 + Q[5] * u2;
    }
    // C b_l(g) of the membrane incompatible-mode columns, then K_ab / K_bb
    // rows with four independent accumulators.
    if (valid) {
        for (int w = tl; w < 16; w += Q4_TEAM) {
            const int g = w >> 2, l = w & 3;
            double b[3];
            q4_bi_col(S.g, g, l, b);
#pragma unroll
            for (int r = 0; r < 3; ++r) S.P[g][l][r] = S.Cm[3 * r] * b[0] + S.Cm[3 * r + 1] * b[1] + S.Cm[3 * r + 2] * b[2];
        }
    }
    __syncwarp();
    if (valid) {
        for (int r = tl; r < 12; r += Q4_TEAM) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                double a[3];
                if (r < 8) q4_mem_col(S.g, g, r >> 1, r & 1, a);
                else q4_bi_col(S.g, g, r - 8, a);
                const double wd = S.g.wdet[g];
#pragma unroll
                for (int l = 0; l < 4; ++l) {
                    const double *P = S.P[g][l];
                    acc[l] += wd * (a[0] * P[0] + a[1] * P[1] + a[2] * P[2]);
                }
            }
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                if (r < 8) S.Kabm[r][l] = acc[l];
                else S.Kbbm[4 * (r - 8) + l] = acc[l];
            }
        }
    }
    __syncwarp();
    if (valid && tl == 0) inv4_inplace(S.Kbbm);
    __syncwarp();
    // condensation map A = -Kbb^-1 Kab' on the membrane dofs
    if (valid) {
        for (int w = tl; w < 32; w += Q4_TEAM) {
            int l = w >> 3, r = w & 7;
            double s = 0.0;
            for (int q = 0; q < 4; ++q) s += S.Kbbm[4 * l + q] * S.Kabm[r][q];
            S.Am[l][r] = -s;
        }
    }
    __syncwarp();
    if (valid && tl < 4) {
        double s = 0.0;
        for (int r = 0; r < 8; ++r) s += S.Am[tl][r] * S.uuv[r];
        S.alpha[tl] = s;
    }
    __syncwarp();
    // Gauss-point stresses, principal directions and gradient vectors:
    // lane tl < 8 handles Gauss point g = tl / 2, principal direction tl % 2.
    if (valid && tl < 8) {
        const int g = tl >> 1, dir = tl & 1;
        const Q4Geo &G = S.g;
        double exx = 0.0, eyy = 0.0, gxy = 0.0;
        for (int k = 0; k < 4; ++k) {
            double x = G.dNx[g][k], y = G.dNy[g][k];
            exx += x * S.uuv[2 * k];
            eyy += y * S.uuv[2 * k + 1];
            gxy += y * S.uuv[2 * k] + x * S.uuv[2 * k + 1];
        }
        double d1x = G.dphi[g][0], d1y = G.dphi[g][1], d2x = G.dphi[g][2], d2y = G.dphi[g][3];
        exx += d1x * S.alpha[0] + d2x * S.alpha[2];
        eyy += d1y * S.alpha[1] + d2y * S.alpha[3];
        gxy += d1y * S.alpha[0] + d1x * S.alpha[1] + d2y * S.alpha[2] + d2x * S.alpha[3];
        double h = S.h;
        double sxx = (S.Cm[0] * exx + S.Cm[1] * eyy + S.Cm[2] * gxy) / h;
        double syy = (S.Cm[3] * exx + S.Cm[4] * eyy + S.Cm[5] * gxy) / h;
        double sxy = (S.Cm[6] * exx + S.Cm[7] * eyy + S.Cm[8] * gxy) / h;
        // principal_stress_2d_components (FEMKernels.jl:6891-6902)
        double mean = 0.5 * (sxx + syy), hd = 0.5 * (sxx - syy);
        double rad = sqrt(hd * hd + sxy * sxy);
        double lam, c, sn;
        if (rad <= 1e-30) {
            lam = mean;
            c = dir == 0 ? 1.0 : 0.0;
            sn = dir == 0 ? 0.0 : 1.0;
        } else {
            // theta = atan2(2 sxy, sxx - syy) / 2 lies in [-pi/2, pi/2], so
            // (cos theta, sin theta) follow from cos 2theta = hd / rad and
            // sin 2theta = sxy / rad by the half-angle identities, taking the
            // square root on the side without cancellation.
            double c1, s1;
            if (hd >= 0.0) {
                c1 = sqrt((rad + hd) / (2.0 * rad));
                s1 = sxy / (2.0 * c1 * rad);
            } else {
                s1 = copysign(sqrt((rad - hd) / (2.0 * rad)), sxy);
                c1 = sxy / (2.0 * s1 * rad);
            }
            if (dir == 0) { lam = mean + rad; c = c1; sn = s1; }
            else { lam = mean - rad; c = -s1; sn = c1; }
        }
        double f = (fabs(lam) <= 1e-30) ? 0.0 : (h * G.wdet[g]) * lam;
        S.f[tl] = f;
        for (int r = 0; r < 8; ++r) {
            int k = r >> 1, comp = r & 1;
            double ux_dx = d1x * S.Am[0][r] + d2x * S.Am[2][r];
            double ux_dy = d1y * S.Am[0][r] + d2y * S.Am[2][r];
            double uy_dx = d1x * S.Am[1][r] + d2x * S.Am[3][r];
            double uy_dy = d1y * S.Am[1][r] + d2y * S.Am[3][r];
            if (comp == 0) { ux_dx += G.dNx[g][k]; ux_dy += G.dNy[g][k]; }
            else { uy_dx += G.dNx[g][k]; uy_dy += G.dNy[g][k]; }
            double gx = c * ux_dx + sn * ux_dy, gy = c * uy_dx + sn * uy_dy;
            S.t[tl][r] = sn * gx - c * gy;
        }
        for (int k = 0; k < 4; ++k) S.gz[tl][k] = c * G.dNx[g][k] + sn * G.dNy[g][k];
    }
    __syncwarp();
    if (valid) {
        const int a = c_pair_a[tl], b = c_pair_b[tl];
        double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            double f = S.f[q];
            double ta0 = S.t[q][2 * a], ta1 = S.t[q][2 * a + 1], tb0 = S.t[q][2 * b], tb1 = S.t[q][2 * b + 1];
            M[0][0] += f * ta0 * tb0; M[0][1] += f * ta0 * tb1;
            M[1][0] += f * ta1 * tb0; M[1][1] += f * ta1 * tb1;
            M[2][2] += f * S.gz[q][a] * S.gz[q][b];
        }
        double O[3][3];
        rot_block(S.g.Q[a], M, S.g.Q[b], O);
        const int32_t sl = __ldg(o.blk_slot + e * 10 + tl);
        const double Z[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        double lmax = 0.0;
        write_sub_block(o, e, sl, a, b, 0, 0, O, lmax, 24);
        write_sub_block(o, e, sl, a, b, 0, 1, Z, lmax, 24);
        write_sub_block(o, e, sl, a, b, 1, 0, Z, lmax, 24);
        write_sub_block(o, e, sl, a, b, 1, 1, Z, lmax, 24);
    }
}

}  // namespace jfg
