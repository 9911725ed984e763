// elem_q4.cuh -- CQUAD4 stiffness (K) and differential stiffness (KG) kernels.
//
// Mapping: a team of 10 lanes owns one element, three teams per warp
// (lanes 30-31 only join the warp barriers).  Every lane of a team computes
// the frame and local coordinates in registers; per-point and per-row
// intermediates are spread over the lanes and meet in shared memory; the
// final phase gives each lane one node pair (a <= b) of the symmetric 24x24
// global matrix, so the 300 packed values are produced without redundant
// work and written straight to their sorted contribution slots
// (deterministic segmented reduction follows).
//
// K follows stiffness_quad4_matrices' default planar branch
// (src/FEMKernels.jl:3185-4034): 2x2 Gauss membrane + bending with the
// MacNeal twist row (:3670-3673), Hughes-Brezzi drilling (:3556-3559,
// :3778-3779), Wilson incompatible modes condensed (:3790-3801, :3964-4011;
// both condensations through one LDL' factorisation, see Q4KShared) and
// MacNeal's residual-bending-flexibility shear (add_quad4_macneal_shear_rbf!,
// :4715-4978); then T'KT with T built from the
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
    bool kg_layout = false;              // KG staging layout (see blk_entry), else K's
    double *kg_rot = nullptr;            // KG: rotation sub-blocks of bar pairs (kKgRotStride doubles per bar pair)

    __device__ __forceinline__ ElemOut at(int v) const {
        ElemOut r = *this;
        r.staging += v * staging_stride;
        r.exc_raw += v * exc_stride;
        if (diag_staging) r.diag_staging += v * dstage_stride;
        if (maxabs) r.maxabs += v;
        if (h) r.h += v * h_stride;
        if (bprop) r.bprop += v * bprop_stride;
        if (kg_rot) r.kg_rot += v * staging_stride;
        return r;
    }
    // Shell thickness of element e: the variant's own, else the property record's.
    __device__ __forceinline__ double thickness(int64_t e, const double *pr) const { return h ? __ldg(h + e) : __ldg(pr); }
};

// KG rotation sub-blocks of a bar pair: 27 values padded to 28 doubles, so
// that every pair's record starts on 16 bytes (one bulk copy per pair).
constexpr int kKgRotStride = 28;

constexpr int32_t kBlkTranspose = 1 << 30;
constexpr int32_t kBlkIndexMask = kBlkTranspose - 1;

// Address of entry (i, j) of a pair block given its slot.  Raw RBE2 blocks
// are row-major 6x6.  K stages 36 values per slot, row-major.  KG stages 12
// values per slot: the translation 3x3 (row-major) and three values of
// padding, so a shell's KG contribution (translations only) fills whole
// 32-byte sectors; the other three 3x3 sub-blocks of a bar pair (translation-
// rotation, rotation-translation, rotation-rotation) go to kg_rot at the bar
// pair's index.
__device__ __forceinline__ double *blk_entry(const ElemOut &o, int32_t s, int i, int j, int64_t bar_pair = 0) {
    if (s < 0) return o.exc_raw + 36 * (int64_t)(-(s + 1)) + 6 * i + j;
    const int64_t idx = s & kBlkIndexMask;
    const int r = (s & kBlkTranspose) ? j : i, c = (s & kBlkTranspose) ? i : j;
    if (!o.kg_layout) return o.staging + 36 * idx + 6 * r + c;
    if (r < 3 && c < 3) return o.staging + 12 * idx + 3 * r + c;
    return o.kg_rot + kKgRotStride * bar_pair + 9 * (2 * (r / 3) + c / 3 - 1) + 3 * (r % 3) + (c % 3);
}

// The padding of a staged KG shell slot (see blk_entry).
__device__ __forceinline__ void kg_shell_pad(const ElemOut &o, int32_t s) {
    if (s < 0) return;
    double *base = o.staging + 12 * (int64_t)(s & kBlkIndexMask);
    base[9] = 0.0; base[10] = 0.0; base[11] = 0.0;
}

// Per-point data of one CQUAD4 shared by its team.
struct Q4Pts {
    double dNx[5][4], dNy[5][4];  // 4 Gauss points + centre (index 4)
    double wdet[4];
    double dphi[4][4];            // d1x, d1y, d2x, d2y per Gauss point
};

// K kernel state of one element.  The isotropic constitutive matrices are
// scalar multiples of one plane-stress matrix P(nu): Cm = cm P, Cb = cb P.
// The incompatible-mode blocks therefore factor as K_ab = cm Am, K_bb = cm B
// (membrane) and K_abb = cb Ab S, K_bbb = cb S' B S (bending), where Am, Ab
// and B hold geometry and P only and S is the signed permutation taking the
// bending modes (-m1, -m3, m0, m2) to the membrane modes m0..m3.  Both
// condensations K_ab K_bb^-1 K_ab' are then c A B^-1 A' with the one 4x4
// symmetric positive definite B.
struct __align__(16) Q4KShared {
    union {
        struct {
            Q4Pts g;
            double Dd[4][4];            // MacNeal sampling rows: dN_k/dx (rows 0, 1), dN_k/dy (rows 2, 3)
            double ivd[4];              // 1 / (sqrt(2 Jp)^2 cs) per sampling point
            double W[6];                // Zx^-1 (w00, w01, w11), Zy^-1 (w22, w23, w33)
            double Am[8][4], Ab[8][4];  // rows: (node, component) of the membrane / bending B
            double B[10];               // packed upper triangle
            double Xm[4][8], Xb[4][8];  // B^-1 Am', B^-1 Ab'
        };
        // write phase: the element's rotated pair blocks, stored orientation, each
        // padded to 38 doubles: the 16-byte staging stores of a warp's 30 lanes
        // then spread over all eight 16-byte bank groups (36 would use four)
        double blk[10][38];
    };
};

// KG kernel state of one element (membrane incompatible modes only; the
// condensation map is -B^-1 Am' with Am, B as in the K kernel).
struct __align__(16) Q4GShared {
    Q4Pts g;
    double uuv[8];        // local (u, v) of each node
    double Am[8][4];
    double B[10];
    double map[4][8];     // -B^-1 Am'
    alignas(16) double t[8][8];  // (node, component) pairs adjacent: read as 16-byte pairs
    double gz[8][4], f[8];
};
static_assert(sizeof(Q4GShared) >= 10 * 14 * sizeof(double), "the KG write phase stages ten 14-double slots in the record");

__device__ __forceinline__ void q4_shape_gp(int g, double &r, double &s) {
    const double pt = 0.57735026918962576451;  // 1/sqrt(3)
    r = (g == 0 || g == 3) ? -pt : pt;
    s = (g <= 1) ? -pt : pt;
}

__device__ __forceinline__ double q4_N(int k, double r, double s) {
    return 0.25 * (1 + ((k == 1 || k == 2) ? r : -r)) * (1 + (k >= 2 ? s : -s));
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

// Element frame (q4_frame) and corner coordinates about the centroid
// (assembly.jl:2693-2698), in registers.
__device__ __forceinline__ void q4_local(const double p[4][3], double V[9], double lc[4][2]) {
    double v1[3], v2[3], v3[3];
    q4_frame(p[0], p[1], p[2], p[3], v1, v2, v3);
    double c[3];
    for (int i = 0; i < 3; ++i) c[i] = (p[0][i] + p[1][i] + p[2][i] + p[3][i]) / 4.0;
    for (int k = 0; k < 4; ++k) {
        double d[3];
        sub3(p[k], c, d);
        lc[k][0] = dot3(d, v1);
        lc[k][1] = dot3(d, v2);
    }
    for (int i = 0; i < 3; ++i) { V[i] = v1[i]; V[3 + i] = v2[i]; V[6 + i] = v3[i]; }
}

// Natural coordinates of point pt: 0-3 the 2x2 Gauss points, 4 the centre,
// 5-8 MacNeal's strain-sampling points (0, -p), (0, p), (-p, 0), (p, 0).
__device__ __forceinline__ void q4_point_rs(int pt, double &r, double &s) {
    const double p = 0.57735026918962576451;  // 1/sqrt(3)
    r = pt < 4 ? ((pt == 0 || pt == 3) ? -p : p) : (pt == 7 ? -p : (pt == 8 ? p : 0.0));
    s = pt < 4 ? (pt <= 1 ? -p : p) : (pt == 5 ? -p : (pt == 6 ? p : 0.0));
}

// Shape-function derivatives at (r, s): returns det J (clamped away from 0
// to +-1e-14 when `clamp`, as the MacNeal sampling does) and writes
// dN/dx, dN/dy and the inverse Jacobian (iJ11, iJ12, iJ21, iJ22).
__device__ __forceinline__ double q4_point_derivs(const double lc[4][2], double r, double s, bool clamp,
                                                  double dx[4], double dy[4], double iJ[4]) {
    const double dNr[4] = {-0.25 * (1 - s), 0.25 * (1 - s), 0.25 * (1 + s), -0.25 * (1 + s)};
    const double dNs[4] = {-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r), 0.25 * (1 - r)};
    double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        J11 += dNr[k] * lc[k][0]; J12 += dNr[k] * lc[k][1];
        J21 += dNs[k] * lc[k][0]; J22 += dNs[k] * lc[k][1];
    }
    double det = J11 * J22 - J12 * J21;
    if (clamp && fabs(det) < 1e-14) det = det < 0.0 ? -1e-14 : 1e-14;
    const double inv = 1.0 / det;
    iJ[0] = J22 * inv; iJ[1] = -J12 * inv; iJ[2] = -J21 * inv; iJ[3] = J11 * inv;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        dx[k] = iJ[0] * dNr[k] + iJ[1] * dNs[k];
        dy[k] = iJ[2] * dNr[k] + iJ[3] * dNs[k];
    }
    return det;
}

// Node pair (a <= b) of team lane tl: (0,0) (0,1) (0,2) (0,3) (1,1) (1,2)
// (1,3) (2,2) (2,3) (3,3).
__device__ __forceinline__ void q4_pair(int tl, int &a, int &b) {
    a = (tl >= 4) + (tl >= 7) + (tl >= 9);
    b = a + tl - (a == 0 ? 0 : (a == 1 ? 4 : (a == 2 ? 7 : 9)));
}

// Out = Qa' M Qb for a 3x3 block M whose structural zeros are the clear bits
// of NZ (bit 3 r + c set when M[r][c] may be nonzero).
template <int NZ>
__device__ __forceinline__ void rot_sparse(const double *Qa, const double M[3][3], const double *Qb, double out[3][3]) {
    double W[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double w = 0.0;
            bool any = false;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if ((NZ >> (3 * r + c)) & 1) { w = any ? w + M[r][c] * Qb[3 * c + j] : M[r][c] * Qb[3 * c + j]; any = true; }
            W[r][j] = w;
        }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double o = 0.0;
            bool any = false;
#pragma unroll
            for (int r = 0; r < 3; ++r)
                if ((NZ >> (3 * r)) & 7) { o = any ? o + Qa[3 * r + i] * W[r][j] : Qa[3 * r + i] * W[r][j]; any = true; }
            out[i][j] = o;
        }
}

// Solve B x = rhs with the LDL' factors of the packed SPD 4x4 B.
struct Ldl4 {
    double l10, l20, l30, l21, l31, l32, r0, r1, r2, r3;
    // The first three pivots are ratios of leading principal minors,
    // d0 = m1, d1 = m2 / m1, d2 = m3 / m2, so their reciprocals come from one
    // division, 1 / (m1 m2 m3), instead of a chain of three.
    __device__ __forceinline__ explicit Ldl4(const double *B) {
        const double b00 = B[0], b01 = B[1], b02 = B[2], b03 = B[3], b11 = B[4], b12 = B[5], b13 = B[6];
        const double b22 = B[7], b23 = B[8], b33 = B[9];
        const double m1 = b00, m2 = b00 * b11 - b01 * b01;
        const double m3 = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) + b02 * (b01 * b12 - b11 * b02);
        const double R = 1.0 / (m1 * m2 * m3);
        r0 = (m2 * m3) * R;
        r1 = m1 * ((m1 * m3) * R);
        r2 = m2 * ((m1 * m2) * R);
        l10 = b01 * r0; l20 = b02 * r0; l30 = b03 * r0;
        const double u12 = b12 - l10 * b02, u13 = b13 - l10 * b03;
        l21 = u12 * r1; l31 = u13 * r1;
        const double u23 = b23 - l20 * b03 - l21 * u13;
        l32 = u23 * r2;
        r3 = 1.0 / (b33 - l30 * b03 - l31 * u13 - l32 * u23);
    }
    __device__ __forceinline__ void solve(const double rhs[4], double x[4]) const {
        const double y0 = rhs[0], y1 = rhs[1] - l10 * y0, y2 = rhs[2] - l20 * y0 - l21 * y1;
        const double y3 = rhs[3] - l30 * y0 - l31 * y1 - l32 * y2;
        x[3] = y3 * r3;
        x[2] = y2 * r2 - l32 * x[3];
        x[1] = y1 * r1 - l21 * x[2] - l31 * x[3];
        x[0] = y0 * r0 - l10 * x[1] - l20 * x[2] - l30 * x[3];
    }
};

// MacNeal residual-bending-flexibility scalars of one (virtual) quad with
// corner coordinates lc and isotropic bending stiffness cb
// (add_quad4_macneal_shear_rbf!, FEMKernels.jl:4803-4869: eps 0.04, zb 0.65,
// flex 1/Cb11 = 1/Cb22): zs = (zxu + zxd, zxu - zxd, zyu + zyd, zyu - zyd).
__device__ __forceinline__ void macneal_zs(const double lc[4][2], double cb, double zs[4]) {
    const double Dx = 0.5 * (lc[1][0] + lc[2][0] - lc[0][0] - lc[3][0]);
    const double Dy = 0.5 * (lc[2][1] + lc[3][1] - lc[0][1] - lc[1][1]);
    const double Dx2 = Dx * Dx, Dy2 = Dy * Dy;
    const double J11c = 0.25 * (-lc[0][0] + lc[1][0] + lc[2][0] - lc[3][0]);
    const double J12c = 0.25 * (-lc[0][1] + lc[1][1] + lc[2][1] - lc[3][1]);
    const double J21c = 0.25 * (-lc[0][0] - lc[1][0] + lc[2][0] + lc[3][0]);
    const double J22c = 0.25 * (-lc[0][1] - lc[1][1] + lc[2][1] + lc[3][1]);
    const double A_elem = 4.0 * fabs(J11c * J22c - J12c * J21c);
    const double eps = 0.04;
    // ap = eps / (eps + (1 - eps) Dx2 / Dy2) and bp likewise, each as one
    // quotient; c12 * flex = 0.65 / (12 A_elem) / |cb| as one quotient
    const double dy2 = fmax(Dy2, 1e-30), dx2 = fmax(Dx2, 1e-30);
    const double ap = (eps * dy2) / (eps * dy2 + (1.0 - eps) * Dx2);
    const double bp = (eps * dx2) / (eps * dx2 + (1.0 - eps) * Dy2);
    const double cf = 0.65 / (12.0 * A_elem * fmax(fabs(cb), 1e-30));
    const double zxu = cf * Dx2, zxd = cf * ap * Dx2;
    const double zyu = cf * Dy2, zyd = cf * bp * Dy2;
    zs[0] = zxu + zxd; zs[1] = zxu - zxd; zs[2] = zyu + zyd; zs[3] = zyu - zyd;
}

// 1 / (sqrt(2 |det J|)^2 cs) at a strain-sampling point (V G V of the
// reference with an isotropic shear matrix cs I, floored at 1e-30).
__device__ __forceinline__ double macneal_ivd(double det, double cs) {
    const double sq = sqrt(2.0 * fabs(det));
    const double v = sq * sq * cs;
    return 1.0 / (v < 1e-30 ? 1e-30 : v);
}

// Z = sym(inv(VGV) + Zb) is block diagonal with 2x2 blocks on the
// xi-sampling rows (0, 1) and the eta-sampling rows (2, 3); W holds the two
// inverse blocks (w00, w01, w11, w22, w23, w33).
__device__ __forceinline__ void macneal_w(const double ivd[4], const double zs[4], double W[6]) {
    const double zx00 = ivd[0] + zs[0], zx11 = ivd[1] + zs[0], zx01 = zs[1];
    const double zy00 = ivd[2] + zs[2], zy11 = ivd[3] + zs[2], zy01 = zs[3];
    const double dx = zx00 * zx11 - zx01 * zx01, dy = zy00 * zy11 - zy01 * zy01;
    const double r = 1.0 / (dx * dy), ix = dy * r, iy = dx * r;  // both inverses from one reciprocal
    W[0] = zx11 * ix; W[1] = -zx01 * ix; W[2] = zx00 * ix;
    W[3] = zy11 * iy; W[4] = -zy01 * iy; W[5] = zy00 * iy;
}

// MacNeal's shear term D_a' Z^-1 D_b of node pair (a, b) on (w, theta_x,
// theta_y), added to P.  D's columns for node k: w -> (dN/dx at the
// xi-sampling rows, dN/dy at the eta-sampling rows), theta_x -> -N on the
// eta rows, theta_y -> N on the xi rows; the theta_x-theta_y coupling is zero.
__device__ __forceinline__ void macneal_pair(const double (*Dd)[4], const double *W, int a, int b, double P[3][3]) {
    const double pt = 0.57735026918962576451;
    const double cxa0 = Dd[0][a], cxa1 = Dd[1][a], cya0 = Dd[2][a], cya1 = Dd[3][a];
    const double cxb0 = Dd[0][b], cxb1 = Dd[1][b], cyb0 = Dd[2][b], cyb1 = Dd[3][b];
    const double nxa0 = q4_N(a, 0.0, -pt), nxa1 = q4_N(a, 0.0, pt);
    const double nya0 = -q4_N(a, -pt, 0.0), nya1 = -q4_N(a, pt, 0.0);
    const double nxb0 = q4_N(b, 0.0, -pt), nxb1 = q4_N(b, 0.0, pt);
    const double nyb0 = -q4_N(b, -pt, 0.0), nyb1 = -q4_N(b, pt, 0.0);
    const double w0 = W[0], w1 = W[1], w2 = W[2], w3 = W[3], w4 = W[4], w5 = W[5];
    const double yx0 = w0 * cxb0 + w1 * cxb1, yx1 = w1 * cxb0 + w2 * cxb1;
    const double ynx0 = w0 * nxb0 + w1 * nxb1, ynx1 = w1 * nxb0 + w2 * nxb1;
    const double yy0 = w3 * cyb0 + w4 * cyb1, yy1 = w4 * cyb0 + w5 * cyb1;
    const double yny0 = w3 * nyb0 + w4 * nyb1, yny1 = w4 * nyb0 + w5 * nyb1;
    P[0][0] += (cxa0 * yx0 + cxa1 * yx1) + (cya0 * yy0 + cya1 * yy1);
    P[0][1] += cya0 * yny0 + cya1 * yny1;
    P[0][2] += cxa0 * ynx0 + cxa1 * ynx1;
    P[1][0] += nya0 * yy0 + nya1 * yy1;
    P[1][1] += nya0 * yny0 + nya1 * yny1;
    P[2][0] += nxa0 * yx0 + nxa1 * yx1;
    P[2][2] += nxa0 * ynx0 + nxa1 * ynx1;
}

// Bending stiffness with the MacNeal twist row (0, -y, 2(-x) + xc) /
// (x, 0, 2y - yc) for node pair (a, b) over the 2x2 Gauss points, isotropic
// Cb = cb P(nu): the (theta_x, theta_y) 2x2 block added to P[1..2][1..2].
__device__ __forceinline__ void bend_pair(const double (*dNx)[4], const double (*dNy)[4], const double *wdet, int a, int b,
                                          double cb, double nu, double gam, double P[3][3]) {
    double Pxx = 0, Pxy = 0, Pyx = 0, Pyy = 0, T00 = 0, T01 = 0, T10 = 0, T11 = 0;
    const double xca = dNx[4][a], yca = dNy[4][a], xcb = dNx[4][b], ycb = dNy[4][b];
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        const double wd = wdet[g];
        const double xa = dNx[g][a], ya = dNy[g][a], xb = dNx[g][b], yb = dNy[g][b];
        const double t0a = 2.0 * (-xa) - (-xca), t1a = 2.0 * ya - yca;
        const double t0b = 2.0 * (-xb) - (-xcb), t1b = 2.0 * yb - ycb;
        const double wx = wd * xa, wy = wd * ya, w0 = wd * t0a, w1 = wd * t1a;
        Pxx += wx * xb; Pxy += wx * yb; Pyx += wy * xb; Pyy += wy * yb;
        T00 += w0 * t0b; T01 += w0 * t1b; T10 += w1 * t0b; T11 += w1 * t1b;
    }
    P[1][1] += cb * (Pyy + gam * T00);
    P[1][2] += cb * (gam * T01 - nu * Pyx);
    P[2][1] += cb * (gam * T10 - nu * Pxy);
    P[2][2] += cb * (Pxx + gam * T11);
}

// W warps per CTA (3 W elements): 4 or 8.  The element records are dynamic
// shared memory, Q4_TEAMS_PER_WARP * W * sizeof(Q4KShared) bytes.
template <int W>
__global__ void __launch_bounds__(32 * W, 16 / W) q4_k_kernel(int64_t nq, const int32_t *__restrict__ nodes,
                                                         const double *__restrict__ prop,
                                                         const double *__restrict__ coords,
                                                         const double *__restrict__ nodeR, double k6rot, ElemOut o) {
    extern __shared__ __align__(16) unsigned char q4_smem[];
    Q4KShared *sh = reinterpret_cast<Q4KShared *>(q4_smem);
    o = o.at(blockIdx.y);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane / Q4_TEAM, tl = lane - team * Q4_TEAM;
    const bool in_team = team < Q4_TEAMS_PER_WARP;
    const int slot_id = warp * Q4_TEAMS_PER_WARP + (in_team ? team : 0);
    const int64_t e = (int64_t)blockIdx.x * Q4_TEAMS_PER_WARP * W + slot_id;
    const bool valid = in_team && e < nq;
    Q4KShared &S = sh[slot_id];

    // Phase 0, every lane of the team in registers: nodes, corners,
    // property record, frame, local coordinates and the constitutive scalars
    // of isotropic PSHELL/MAT1 (assembly.jl:2460-2469).
    int nd[4] = {0, 0, 0, 0};
    double V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double lc[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    double h = 1.0, E = 0.0, nu = 0.0, br = 0.0, tst = 0.0, Gs = 0.0;
    if (valid) {
        const double *pr = prop + 7 * e;
        h = o.thickness(e, pr); E = __ldg(pr + 1); nu = __ldg(pr + 2); br = __ldg(pr + 4); tst = __ldg(pr + 5);
        Gs = __ldg(pr + 6);
#pragma unroll
        for (int k = 0; k < 4; ++k) nd[k] = __ldg(nodes + 4 * e + k);
        double p[4][3];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
        q4_local(p, V, lc);
    }
    const double gam = (1 - nu) / 2;
    const double inu = 1.0 / (1 - nu * nu);  // one reciprocal for cm, cb and G_drill
    const double cm = E * h * inu;
    const double cb = br * (E * h * h * h) * (inu * (1.0 / 12.0));
    const bool membrane_only = br <= 1e-12;
    const double cs = membrane_only ? 0.0 : tst * h * Gs;
    double G_drill = E * inu * gam;  // Cm33 / h
    if (G_drill < 1e-6) G_drill = E / (2 * 3.0);
    const double ad = membrane_only ? 0.0 : (k6rot / 1e5) * G_drill * h;
    const bool skip_mac = h < 1e-30 || fabs(cs) < 1e-30;

    // Phase 1: point derivatives (lanes 0-8), MacNeal element scalars (lane 9).
    double zs[4] = {0.0, 0.0, 0.0, 0.0};  // zxu + zxd, zxu - zxd, zyu + zyd, zyu - zyd
    if (valid && tl < 9) {
        double r, s, dx[4], dy[4], iJ[4];
        q4_point_rs(tl, r, s);
        const bool mac = tl >= 5;
        const double det = q4_point_derivs(lc, r, s, mac, dx, dy, iJ);
        if (!mac) {
#pragma unroll
            for (int k = 0; k < 4; ++k) { S.g.dNx[tl][k] = dx[k]; S.g.dNy[tl][k] = dy[k]; }
            if (tl < 4) {
                const double a = fabs(det);
                S.g.wdet[tl] = a < 1e-12 ? 1e-12 : a;
                S.g.dphi[tl][0] = iJ[0] * (-2.0 * r);
                S.g.dphi[tl][1] = iJ[2] * (-2.0 * r);
                S.g.dphi[tl][2] = iJ[1] * (-2.0 * s);
                S.g.dphi[tl][3] = iJ[3] * (-2.0 * s);
            }
        } else {
            const int l = tl - 5;
#pragma unroll
            for (int k = 0; k < 4; ++k) S.Dd[l][k] = l < 2 ? dx[k] : dy[k];
            S.ivd[l] = macneal_ivd(det, cs);
        }
    } else if (valid && tl == 9) {
        macneal_zs(lc, cb, zs);
    }
    __syncwarp();

    // Phase 2: rows of Am and Ab (lanes 0-7), B (lane 8), Z^-1 (lane 9).
    double am[4] = {0.0, 0.0, 0.0, 0.0}, ab[4] = {0.0, 0.0, 0.0, 0.0};
    if (valid && tl < 8) {
        const int k = tl >> 1;
        const bool c1 = tl & 1;
        const double xc = S.g.dNx[4][k], yc = S.g.dNy[4][k];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const double wd = S.g.wdet[g], x = S.g.dNx[g][k], y = S.g.dNy[g][k];
            const double d1x = S.g.dphi[g][0], d1y = S.g.dphi[g][1], d2x = S.g.dphi[g][2], d2y = S.g.dphi[g][3];
            // membrane column (x, 0, y) / (0, y, x); bending column with the
            // MacNeal twist row (0, -y, 2(-x) + xc) / (x, 0, 2y - yc)
            const double m0 = wd * (c1 ? 0.0 : x), m1 = wd * (c1 ? y : 0.0), m2 = wd * (c1 ? x : y);
            const double t = c1 ? 2.0 * y - yc : 2.0 * (-x) - (-xc);
            const double b0 = wd * (c1 ? x : 0.0), b1 = wd * (c1 ? 0.0 : -y), b2 = wd * t;
            const double P[4][3] = {{d1x, nu * d1x, gam * d1y}, {nu * d1y, d1y, gam * d1x},
                                    {d2x, nu * d2x, gam * d2y}, {nu * d2y, d2y, gam * d2x}};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                am[m] += m0 * P[m][0] + m1 * P[m][1] + m2 * P[m][2];
                ab[m] += b0 * P[m][0] + b1 * P[m][1] + b2 * P[m][2];
            }
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) { S.Am[tl][m] = am[m]; S.Ab[tl][m] = ab[m]; }
    } else if (valid && tl == 8) {
        double Bs[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const double wd = S.g.wdet[g];
            const double d1x = S.g.dphi[g][0], d1y = S.g.dphi[g][1], d2x = S.g.dphi[g][2], d2y = S.g.dphi[g][3];
            const double P[4][3] = {{d1x, nu * d1x, gam * d1y}, {nu * d1y, d1y, gam * d1x},
                                    {d2x, nu * d2x, gam * d2y}, {nu * d2y, d2y, gam * d2x}};
            // modes m0 = (d1x, 0, d1y), m1 = (0, d1y, d1x), m2 = (d2x, 0, d2y), m3 = (0, d2y, d2x)
            Bs[0] += wd * (d1x * P[0][0] + d1y * P[0][2]);
            Bs[1] += wd * (d1x * P[1][0] + d1y * P[1][2]);
            Bs[2] += wd * (d1x * P[2][0] + d1y * P[2][2]);
            Bs[3] += wd * (d1x * P[3][0] + d1y * P[3][2]);
            Bs[4] += wd * (d1y * P[1][1] + d1x * P[1][2]);
            Bs[5] += wd * (d1y * P[2][1] + d1x * P[2][2]);
            Bs[6] += wd * (d1y * P[3][1] + d1x * P[3][2]);
            Bs[7] += wd * (d2x * P[2][0] + d2y * P[2][2]);
            Bs[8] += wd * (d2x * P[3][0] + d2y * P[3][2]);
            Bs[9] += wd * (d2y * P[3][1] + d2x * P[3][2]);
        }
#pragma unroll
        for (int i = 0; i < 10; ++i) S.B[i] = Bs[i];
    } else if (valid && tl == 9 && !skip_mac) {
        macneal_w(S.ivd, zs, S.W);
    }
    __syncwarp();

    // Phase 3: X = B^-1 A' for both condensations, one A row per lane.
    if (valid && tl < 8) {
        const Ldl4 f(S.B);
        double x[4];
        f.solve(am, x);
#pragma unroll
        for (int l = 0; l < 4; ++l) S.Xm[l][tl] = x[l];
        f.solve(ab, x);
#pragma unroll
        for (int l = 0; l < 4; ++l) S.Xb[l][tl] = x[l];
    }
    __syncwarp();

    // Phase 4: one node pair (a <= b) per lane.  Gauss-point sums and the
    // 6x6 local block (18 structural nonzeros).
    double lmax = 0.0;
    int a = 0, b = 0;
    int32_t sl = -1;
    double Lm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Lp[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double Qa[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Qb[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (valid) {
        q4_pair(tl, a, b);
        double Pxx = 0, Pxy = 0, Pyx = 0, Pyy = 0, T00 = 0, T01 = 0, T10 = 0, T11 = 0;
        double SxN = 0, SyN = 0, SNx = 0, SNy = 0, SNN = 0;
        const double xca = S.g.dNx[4][a], yca = S.g.dNy[4][a], xcb = S.g.dNx[4][b], ycb = S.g.dNy[4][b];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            double r, s;
            q4_shape_gp(g, r, s);
            const double wd = S.g.wdet[g];
            const double xa = S.g.dNx[g][a], ya = S.g.dNy[g][a], xb = S.g.dNx[g][b], yb = S.g.dNy[g][b];
            const double t0a = 2.0 * (-xa) - (-xca), t1a = 2.0 * ya - yca;
            const double t0b = 2.0 * (-xb) - (-xcb), t1b = 2.0 * yb - ycb;
            const double Na = q4_N(a, r, s), Nb = q4_N(b, r, s);
            const double wx = wd * xa, wy = wd * ya, w0 = wd * t0a, w1 = wd * t1a, wn = wd * Na;
            Pxx += wx * xb; Pxy += wx * yb; Pyx += wy * xb; Pyy += wy * yb;
            T00 += w0 * t0b; T01 += w0 * t1b; T10 += w1 * t0b; T11 += w1 * t1b;
            SxN += wx * Nb; SyN += wy * Nb; SNx += wn * xb; SNy += wn * yb; SNN += wn * Nb;
        }
        // incompatible-mode condensations
        double cmm[2][2], cbb[2][2];
#pragma unroll
        for (int al = 0; al < 2; ++al)
#pragma unroll
            for (int be = 0; be < 2; ++be) {
                double sm = 0.0, sb = 0.0;
#pragma unroll
                for (int l = 0; l < 4; ++l) {
                    sm += S.Am[2 * a + al][l] * S.Xm[l][2 * b + be];
                    sb += S.Ab[2 * a + al][l] * S.Xb[l][2 * b + be];
                }
                cmm[al][be] = sm;
                cbb[al][be] = sb;
            }
        // membrane + drilling on (u, v, theta_z): Bd = (dN/dy / 2, -dN/dx / 2, N)
        const double q = 0.25 * ad, hq = 0.5 * ad;
        Lm[0][0] = cm * (Pxx + gam * Pyy) + q * Pyy - cm * cmm[0][0];
        Lm[0][1] = cm * (nu * Pxy + gam * Pyx) - q * Pyx - cm * cmm[0][1];
        Lm[1][0] = cm * (nu * Pyx + gam * Pxy) - q * Pxy - cm * cmm[1][0];
        Lm[1][1] = cm * (Pyy + gam * Pxx) + q * Pxx - cm * cmm[1][1];
        Lm[0][2] = hq * SyN; Lm[1][2] = -hq * SxN;
        Lm[2][0] = hq * SNy; Lm[2][1] = -hq * SNx; Lm[2][2] = ad * SNN;
        // plate on (w, theta_x, theta_y): bending with the twist row, then
        // MacNeal's shear D' Z^-1 D
        Lp[1][1] = cb * (Pyy + gam * T00) - cb * cbb[0][0];
        Lp[1][2] = cb * (gam * T01 - nu * Pyx) - cb * cbb[0][1];
        Lp[2][1] = cb * (gam * T10 - nu * Pxy) - cb * cbb[1][0];
        Lp[2][2] = cb * (Pxx + gam * T11) - cb * cbb[1][1];
        if (!skip_mac) macneal_pair(S.Dd, S.W, a, b, Lp);
        if (nodeR) {
            double Ra[9], Rb[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                Ra[i] = __ldg(nodeR + 9 * (int64_t)nd[a] + i);
                Rb[i] = __ldg(nodeR + 9 * (int64_t)nd[b] + i);
            }
            node_block(V, V + 3, V + 6, Ra, Qa);
            node_block(V, V + 3, V + 6, Rb, Qb);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) { Qa[i] = V[i]; Qb[i] = V[i]; }
        }
        sl = __ldg(o.blk_slot + e * 10 + tl);
    }
    // Phase 5: T'KT and the writes.  The block of a pair is stored with
    // rows of the lower-numbered global node (transposed when the slot says
    // so).  Each half (stored rows 0-2, then 3-5) is rotated by sub-blocks
    // and staged in the element's shared record -- no lane reads the phase
    // data any more -- which then holds the element's ten 6x6 blocks.  Each
    // lane then copies its own slot out as one 288-byte bulk copy, so a slot
    // is written as whole contiguous lines instead of 36 scattered 8-byte
    // stores.  Pairs on the RBE2 path are written directly.
    __syncwarp();
    const bool t = valid && sl >= 0 && (sl & kBlkTranspose);
    double *buf = S.blk[valid ? tl : 0];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        if (valid) {
            // local dof order (u, v, w, theta_x, theta_y, theta_z); the
            // translation-rotation and rotation-translation sub-blocks share
            // one zero pattern, the two diagonal sub-blocks another
            double M[3][3], Of[3][3], Os[3][3];
            const bool off_tr = (half == 0) != t;  // off-diagonal sub-block of this half: TR, else RT
            M[0][2] = off_tr ? Lm[0][2] : Lp[1][0]; M[1][2] = off_tr ? Lm[1][2] : Lp[2][0];
            M[2][0] = off_tr ? Lp[0][1] : Lm[2][0]; M[2][1] = off_tr ? Lp[0][2] : Lm[2][1];
            if (half == 0) {
                rot_sparse<0b011100100>(Qa, M, Qb, Os);
                M[0][0] = Lm[0][0]; M[0][1] = Lm[0][1]; M[1][0] = Lm[1][0]; M[1][1] = Lm[1][1]; M[2][2] = Lp[0][0];
                rot_sparse<0b100011011>(Qa, M, Qb, Of);
            } else {
                rot_sparse<0b011100100>(Qa, M, Qb, Of);
                M[0][0] = Lp[1][1]; M[0][1] = Lp[1][2]; M[1][0] = Lp[2][1]; M[1][1] = Lp[2][2]; M[2][2] = Lm[2][2];
                rot_sparse<0b100011011>(Qa, M, Qb, Os);
            }
            if (sl < 0) {
                write_sub_block(o, e, sl, a, b, half, 0, Of, lmax, 24);
                write_sub_block(o, e, sl, a, b, half, 1, Os, lmax, 24);
            } else {
                double2 *hb = reinterpret_cast<double2 *>(buf + 18 * half);  // stored row r: 3 pairs
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    double v[6];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        v[c] = t ? Of[c][r] : Of[r][c];
                        v[3 + c] = t ? Os[c][r] : Os[r][c];
                    }
#pragma unroll
                    for (int c = 0; c < 6; ++c) lmax = fmax(lmax, fabs(v[c]));
                    hb[3 * r] = make_double2(v[0], v[1]);
                    hb[3 * r + 1] = make_double2(v[2], v[3]);
                    hb[3 * r + 2] = make_double2(v[4], v[5]);
                }
                if (o.diag_staging && a == b) {
                    // diagonal pair (never transposed): TT in the first, RR in the second column band
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                        o.diag_staging[__ldg(o.diag_slot + e * 24 + 6 * a + 3 * half + i)] = half == 0 ? Of[i][i] : Os[i][i];
                }
            }
        }
    }
    if (valid && sl >= 0) {  // the lane's own staged slot (RBE2-path slots are negative)
        slot_fence();
        slot_copy(o.staging + 36 * (int64_t)(sl & kBlkIndexMask), buf, 288);
    }
    if (o.maxabs) {
        for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
        if (lane == 0 && lmax > 0.0) atomic_max_nonneg(o.maxabs, lmax);
    }
    slot_copies_read();
}

// W warps per CTA (3 W elements): 4 or 8; dynamic shared memory as q4_k_kernel's.
template <int W>
__global__ void __launch_bounds__(32 * W) q4_kg_kernel(int64_t nq, const int32_t *__restrict__ nodes,
                                                          const double *__restrict__ prop,
                                                          const double *__restrict__ coords,
                                                          const double *__restrict__ nodeR,
                                                          const double *__restrict__ u, ElemOut o) {
    extern __shared__ __align__(16) unsigned char q4_smem[];
    Q4GShared *sh = reinterpret_cast<Q4GShared *>(q4_smem);
    o = o.at(blockIdx.y);
    u += (int64_t)blockIdx.y * o.u_stride;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane / Q4_TEAM, tl = lane - team * Q4_TEAM;
    const bool in_team = team < Q4_TEAMS_PER_WARP;
    const int slot_id = warp * Q4_TEAMS_PER_WARP + (in_team ? team : 0);
    const int64_t e = (int64_t)blockIdx.x * Q4_TEAMS_PER_WARP * W + slot_id;
    const bool valid = in_team && e < nq;
    Q4GShared &S = sh[slot_id];

    // Phase 0, every lane in registers: nodes, corners, frame, local
    // coordinates, membrane stiffness scalar.
    int nd[4] = {0, 0, 0, 0};
    double V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double lc[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    double h = 1.0, E = 0.0, nu = 0.0;
    if (valid) {
        const double *pr = prop + 7 * e;
        h = o.thickness(e, pr); E = __ldg(pr + 1); nu = __ldg(pr + 2);
#pragma unroll
        for (int k = 0; k < 4; ++k) nd[k] = __ldg(nodes + 4 * e + k);
        double p[4][3];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
        q4_local(p, V, lc);
    }
    const double gam = (1 - nu) / 2;
    const double rdh = 1.0 / ((1 - nu * nu) * h);  // one reciprocal for cmh and 1/h
    const double cmh = E * h * h * rdh;             // Cm = cmh P(nu)
    const double ih = (1 - nu * nu) * rdh;

    // Phase 1: Gauss-point derivatives (lanes 0-3); local membrane
    // displacements u_elem = T u_global (lanes 4-7, assembly.jl:5176-5185).
    if (valid && tl < 4) {
        double r, s, dx[4], dy[4], iJ[4];
        q4_shape_gp(tl, r, s);
        const double det = q4_point_derivs(lc, r, s, false, dx, dy, iJ);
#pragma unroll
        for (int k = 0; k < 4; ++k) { S.g.dNx[tl][k] = dx[k]; S.g.dNy[tl][k] = dy[k]; }
        const double a = fabs(det);
        S.g.wdet[tl] = a < 1e-12 ? 1e-12 : a;
        S.g.dphi[tl][0] = iJ[0] * (-2.0 * r);
        S.g.dphi[tl][1] = iJ[2] * (-2.0 * r);
        S.g.dphi[tl][2] = iJ[1] * (-2.0 * s);
        S.g.dphi[tl][3] = iJ[3] * (-2.0 * s);
    } else if (valid && tl < 8) {
        const int k = tl - 4;
        double Q[9];
        if (nodeR) {
            double R[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) R[i] = __ldg(nodeR + 9 * (int64_t)nd[k] + i);
            node_block(V, V + 3, V + 6, R, Q);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) Q[i] = V[i];
        }
        const double *ug = u + 6 * (int64_t)nd[k];
        const double u0 = __ldg(ug), u1 = __ldg(ug + 1), u2 = __ldg(ug + 2);
        S.uuv[2 * k] = Q[0] * u0 + Q[1] * u1 + Q[2] * u2;
        S.uuv[2 * k + 1] = Q[3] * u0 + Q[4] * u1 + Q[5] * u2;
    }
    __syncwarp();

    // Phase 2: membrane rows of Am (lanes 0-7) and B (lane 8).
    double am[4] = {0.0, 0.0, 0.0, 0.0};
    if (valid && tl < 8) {
        const int k = tl >> 1;
        const bool c1 = tl & 1;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const double wd = S.g.wdet[g], x = S.g.dNx[g][k], y = S.g.dNy[g][k];
            const double d1x = S.g.dphi[g][0], d1y = S.g.dphi[g][1], d2x = S.g.dphi[g][2], d2y = S.g.dphi[g][3];
            const double m0 = wd * (c1 ? 0.0 : x), m1 = wd * (c1 ? y : 0.0), m2 = wd * (c1 ? x : y);
            const double P[4][3] = {{d1x, nu * d1x, gam * d1y}, {nu * d1y, d1y, gam * d1x},
                                    {d2x, nu * d2x, gam * d2y}, {nu * d2y, d2y, gam * d2x}};
#pragma unroll
            for (int m = 0; m < 4; ++m) am[m] += m0 * P[m][0] + m1 * P[m][1] + m2 * P[m][2];
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) S.Am[tl][m] = am[m];
    } else if (valid && tl == 8) {
        double Bs[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const double wd = S.g.wdet[g];
            const double d1x = S.g.dphi[g][0], d1y = S.g.dphi[g][1], d2x = S.g.dphi[g][2], d2y = S.g.dphi[g][3];
            const double P[4][3] = {{d1x, nu * d1x, gam * d1y}, {nu * d1y, d1y, gam * d1x},
                                    {d2x, nu * d2x, gam * d2y}, {nu * d2y, d2y, gam * d2x}};
            Bs[0] += wd * (d1x * P[0][0] + d1y * P[0][2]);
            Bs[1] += wd * (d1x * P[1][0] + d1y * P[1][2]);
            Bs[2] += wd * (d1x * P[2][0] + d1y * P[2][2]);
            Bs[3] += wd * (d1x * P[3][0] + d1y * P[3][2]);
            Bs[4] += wd * (d1y * P[1][1] + d1x * P[1][2]);
            Bs[5] += wd * (d1y * P[2][1] + d1x * P[2][2]);
            Bs[6] += wd * (d1y * P[3][1] + d1x * P[3][2]);
            Bs[7] += wd * (d2x * P[2][0] + d2y * P[2][2]);
            Bs[8] += wd * (d2x * P[3][0] + d2y * P[3][2]);
            Bs[9] += wd * (d2y * P[3][1] + d2x * P[3][2]);
        }
#pragma unroll
        for (int i = 0; i < 10; ++i) S.B[i] = Bs[i];
    }
    __syncwarp();

    // Phase 3 (lanes 0-7): column tl of the condensation map -B^-1 Am'
    // (quad4_membrane_incompatible_condensation_map, FEMKernels.jl:6708-6785)
    // and, in every one of these lanes, the mode amplitudes
    // alpha = -B^-1 (Am' u) of quad4_membrane_force_field (:6366-6446).
    double alpha[4] = {0.0, 0.0, 0.0, 0.0};
    if (valid && tl < 8) {
        const Ldl4 f(S.B);
        double x[4];
        f.solve(am, x);
#pragma unroll
        for (int l = 0; l < 4; ++l) S.map[l][tl] = -x[l];
        double rhs[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const double ur = S.uuv[r];
#pragma unroll
            for (int l = 0; l < 4; ++l) rhs[l] += S.Am[r][l] * ur;
        }
        f.solve(rhs, x);
#pragma unroll
        for (int l = 0; l < 4; ++l) alpha[l] = -x[l];
    }
    __syncwarp();

    // Phase 4: Gauss-point stresses N/h, principal directions and gradient
    // vectors; lane tl < 8 handles Gauss point g = tl / 2, direction tl % 2.
    if (valid && tl < 8) {
        const int g = tl >> 1, dir = tl & 1;
        double exx = 0.0, eyy = 0.0, gxy = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double x = S.g.dNx[g][k], y = S.g.dNy[g][k], uk = S.uuv[2 * k], vk = S.uuv[2 * k + 1];
            exx += x * uk;
            eyy += y * vk;
            gxy += y * uk + x * vk;
        }
        const double d1x = S.g.dphi[g][0], d1y = S.g.dphi[g][1], d2x = S.g.dphi[g][2], d2y = S.g.dphi[g][3];
        exx += d1x * alpha[0] + d2x * alpha[2];
        eyy += d1y * alpha[1] + d2y * alpha[3];
        gxy += d1y * alpha[0] + d1x * alpha[1] + d2y * alpha[2] + d2x * alpha[3];
        const double sxx = (cmh * (exx + nu * eyy)) * ih;
        const double syy = (cmh * (nu * exx + eyy)) * ih;
        const double sxy = (cmh * (gam * gxy)) * ih;
        // principal_stress_2d_components (FEMKernels.jl:6891-6902)
        const double mean = 0.5 * (sxx + syy), hd = 0.5 * (sxx - syy);
        const double rad = sqrt(hd * hd + sxy * sxy);
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
            // With t = 1 / sqrt(2 rad (rad + |hd|)): for hd >= 0,
            // cos = (rad + hd) t and sin = sxy t; otherwise sin =
            // sign(sxy) (rad - hd) t and cos = |sxy| t.
            double c1, s1;
            const double ah = fabs(hd), t = rsqrt(2.0 * rad * (rad + ah));
            if (hd >= 0.0) {
                c1 = (rad + ah) * t;
                s1 = sxy * t;
            } else {
                s1 = copysign((rad + ah) * t, sxy);
                c1 = fabs(sxy) * t;
            }
            if (dir == 0) { lam = mean + rad; c = c1; sn = s1; }
            else { lam = mean - rad; c = -s1; sn = c1; }
        }
        S.f[tl] = (fabs(lam) <= 1e-30) ? 0.0 : (h * S.g.wdet[g]) * lam;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int k = r >> 1;
            double ux_dx = d1x * S.map[0][r] + d2x * S.map[2][r];
            double ux_dy = d1y * S.map[0][r] + d2y * S.map[2][r];
            double uy_dx = d1x * S.map[1][r] + d2x * S.map[3][r];
            double uy_dy = d1y * S.map[1][r] + d2y * S.map[3][r];
            if ((r & 1) == 0) { ux_dx += S.g.dNx[g][k]; ux_dy += S.g.dNy[g][k]; }
            else { uy_dx += S.g.dNx[g][k]; uy_dy += S.g.dNy[g][k]; }
            const double gx = c * ux_dx + sn * ux_dy, gy = c * uy_dx + sn * uy_dy;
            S.t[tl][r] = sn * gx - c * gy;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) S.gz[tl][k] = c * S.g.dNx[g][k] + sn * S.g.dNy[g][k];
    }
    __syncwarp();

    // Phase 5: one node pair per lane; translations only (the rotation
    // sub-blocks of a flat shell's KG are zero).  A staged slot holds the
    // translation 3x3 and three zeros of padding: each lane stages its slot in
    // the element's shared record and copies it out as one 96-byte bulk copy.
    // Pairs on the RBE2 path are written directly.
    double O[3][3];
    int a = 0, b = 0;
    int32_t sl = -1;
    if (valid) {
        q4_pair(tl, a, b);
        double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const double f = S.f[q];
            const double2 ta = reinterpret_cast<const double2 *>(S.t[q])[a], tb = reinterpret_cast<const double2 *>(S.t[q])[b];
            const double ta0 = ta.x, ta1 = ta.y, tb0 = tb.x, tb1 = tb.y;
            const double fa0 = f * ta0, fa1 = f * ta1;
            M[0][0] += fa0 * tb0; M[0][1] += fa0 * tb1;
            M[1][0] += fa1 * tb0; M[1][1] += fa1 * tb1;
            M[2][2] += (f * S.gz[q][a]) * S.gz[q][b];
        }
        double Qa[9], Qb[9];
        if (nodeR) {
            double Ra[9], Rb[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                Ra[i] = __ldg(nodeR + 9 * (int64_t)nd[a] + i);
                Rb[i] = __ldg(nodeR + 9 * (int64_t)nd[b] + i);
            }
            node_block(V, V + 3, V + 6, Ra, Qa);
            node_block(V, V + 3, V + 6, Rb, Qb);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) { Qa[i] = V[i]; Qb[i] = V[i]; }
        }
        rot_sparse<0b100011011>(Qa, M, Qb, O);
        sl = __ldg(o.blk_slot + e * 10 + tl);
    }
    __syncwarp();  // every lane is past its last read of the element's record
    if (valid) {
        double lmax = 0.0;
        if (sl < 0) {
            // the dof-level RBE2 path reads whole raw blocks; staged shell
            // blocks of KG are read as their translation 3x3 only
            const double Z[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            write_sub_block(o, e, sl, a, b, 0, 0, O, lmax, 24);
            write_sub_block(o, e, sl, a, b, 0, 1, Z, lmax, 24);
            write_sub_block(o, e, sl, a, b, 1, 0, Z, lmax, 24);
            write_sub_block(o, e, sl, a, b, 1, 1, Z, lmax, 24);
        } else {
            const bool t = sl & kBlkTranspose;
            // 14-double stride: the 16-byte stores of a warp's 30 lanes spread
            // over all eight 16-byte bank groups
            double *buf = reinterpret_cast<double *>(&S) + 14 * tl;
            double v[9];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) v[3 * r + c] = t ? O[c][r] : O[r][c];
            double2 *b2 = reinterpret_cast<double2 *>(buf);
            b2[0] = make_double2(v[0], v[1]); b2[1] = make_double2(v[2], v[3]);
            b2[2] = make_double2(v[4], v[5]); b2[3] = make_double2(v[6], v[7]);
            b2[4] = make_double2(v[8], 0.0); b2[5] = make_double2(0.0, 0.0);
            slot_fence();
            slot_copy(o.staging + 12 * (int64_t)(sl & kBlkIndexMask), buf, 96);
        }
    }
    slot_copies_read();
}

}  // namespace jfg
