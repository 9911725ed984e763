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
// and every Kei entry comes from the one quad that holds the corner.  Kii,
// the plate stiffness of the midside and centroid dofs with the corners held,
// is symmetric positive definite, so elimination on the diagonal pivots
// changes only the rounding of the reference's pivoted lu(Kii) \ Kie.  The
// stiffness kernel condenses by 3x3-block elimination (t3_schur); the
// recovery and sensitivity kernels, which need X = Kii^-1 Kie itself, run
// Gauss-Jordan elimination with one row of [Kii | Kie] per lane (t3_condense).
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

struct __align__(16) T3KShared {
    double V[9];
    double R[3][9];  // stiffness kernel: the corners' CD frames, loaded in the set-up phase
    double bv[3], cv[3], A, cm, ad;
    int nd[3];
    union {
        struct {  // virtual-quad data (phases 1-3): Gauss points 0-3, centre 4
            double dNx[3][5][4], dNy[3][5][4], wdet[3][4];
            double Dd[3][4][4], ivd[3][4], zs[3][4], W[3][6];
        } q;
        struct {  // condensation of the recovery and sensitivity kernels
            double X[12][9];   // Kii^-1 Kie
            double Kc[9][9];
        } c;
        struct {  // stiffness kernel, block elimination: Z and diag(d)^-1 Z of each later node
            alignas(16) double Z[6][20];
        } z;
        struct {  // stiffness kernel, write phase: the six 6x6 node-pair blocks as staged,
                  // padded to 38 doubles against shared-memory bank conflicts
            alignas(16) double O[6][38];
        } o;
    } u;
    // recovery and sensitivity kernels: quad q, local node pair (a <= b), 3x3
    // over (w, theta_x, theta_y), padded to 10 doubles.  The stiffness kernel
    // keeps its 28 macro blocks here instead (t3_macro_blocks), padded alike,
    // with one spare block.
    alignas(16) double Pb[3][10][10];
    alignas(16) double Qn[3][10];  // stiffness kernel: each corner's node block T R_k (t3_schur)
    int32_t slot[6];
};

// A 3x3 block (9 doubles) at a 16-byte boundary as 128-bit shared-memory
// accesses: the stiffness kernel's blocks are padded to 10 doubles for this.
__device__ __forceinline__ void ld9(const double *p, double v[9]) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 a = q[0], b = q[1], c = q[2], d = q[3];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y; v[6] = d.x; v[7] = d.y; v[8] = p[8];
}
__device__ __forceinline__ void st9(double *p, const double v[9]) {
    double2 *q = reinterpret_cast<double2 *>(p);
    q[0] = make_double2(v[0], v[1]); q[1] = make_double2(v[2], v[3]);
    q[2] = make_double2(v[4], v[5]); q[3] = make_double2(v[6], v[7]);
    p[8] = v[8];
}

// Corner coordinates of virtual quad q (corner q, midpoint to the next
// corner, centroid, midpoint from the previous corner), as the macro points
// (x_i + x_j) / 2 and (x_0 + x_1 + x_2) / 3 of tria3_plate_macro_data (the
// thirds as a product with 1/3, no division on the points' path).
__device__ __forceinline__ void t3_quad_coords(int q, const double x[3], const double y[3], double lq[4][2]) {
    const int n = q == 2 ? 0 : q + 1, pv = q == 0 ? 2 : q - 1;
    const double xc = q == 0 ? x[0] : (q == 1 ? x[1] : x[2]), yc = q == 0 ? y[0] : (q == 1 ? y[1] : y[2]);
    const double xn = n == 0 ? x[0] : (n == 1 ? x[1] : x[2]), yn = n == 0 ? y[0] : (n == 1 ? y[1] : y[2]);
    const double xp = pv == 0 ? x[0] : (pv == 1 ? x[1] : x[2]), yp = pv == 0 ? y[0] : (pv == 1 ? y[1] : y[2]);
    lq[0][0] = xc; lq[0][1] = yc;
    lq[1][0] = (xc + xn) / 2; lq[1][1] = (yc + yn) / 2;
    lq[2][0] = (x[0] + x[1] + x[2]) * (1.0 / 3.0); lq[2][1] = (y[0] + y[1] + y[2]) * (1.0 / 3.0);
    lq[3][0] = (xp + xc) / 2; lq[3][1] = (yp + yc) / 2;
}

// Plate phases of the CTRIA3 kernels (team of 16 lanes, mask tm), shared by
// the stiffness and the thickness-sensitivity kernels.

// Virtual-quad point data and the MacNeal compliance blocks W of each quad.
__device__ __forceinline__ void t3_plate_points(T3KShared &S, int tl, unsigned tm, const double x[3], const double y[3],
                                                double cs, double cb, bool macneal) {
    // Phase 1: virtual-quad points (27 items: quad q = it / 9, point
    // it % 9 -- Gauss points, centre, MacNeal sampling points) and the
    // MacNeal scalars of each quad (items 27-29).
    for (int it = tl; it < 30; it += T3_TEAM) {
        const int q = it < 27 ? it / 9 : it - 27, pt = it - 9 * (it / 9);
        double lq[4][2];
        t3_quad_coords(q, x, y, lq);
        if (it < 27) {
            double r, s, dx[4], dy[4], iJ[4];
            q4_point_rs(pt, r, s);
            const bool mac = pt >= 5;
            const double det = q4_point_derivs(lq, r, s, mac, dx, dy, iJ);
            if (!mac) {
#pragma unroll
                for (int k = 0; k < 4; ++k) { S.u.q.dNx[q][pt][k] = dx[k]; S.u.q.dNy[q][pt][k] = dy[k]; }
                if (pt < 4) { const double a = fabs(det); S.u.q.wdet[q][pt] = a < 1e-12 ? 1e-12 : a; }
            } else {
                const int l = pt - 5;
#pragma unroll
                for (int k = 0; k < 4; ++k) S.u.q.Dd[q][l][k] = l < 2 ? dx[k] : dy[k];
                S.u.q.ivd[q][l] = macneal_ivd(det, cs);
            }
        } else {
            double zs[4];
            macneal_zs(lq, cb, zs);
#pragma unroll
            for (int i = 0; i < 4; ++i) S.u.q.zs[q][i] = zs[i];
        }
    }
    __syncwarp(tm);
    if (macneal && tl < 3) macneal_w(S.u.q.ivd[tl], S.u.q.zs[tl], S.u.q.W[tl]);
    __syncwarp(tm);
}

// Plate 3x3 block of every (virtual quad, node pair) into S.Pb.
__device__ __forceinline__ void t3_plate_blocks(T3KShared &S, int tl, unsigned tm, double cb, double nu, double gam,
                                                bool macneal) {
    // Phase 2: plate 3x3 block of every (virtual quad, node pair):
    // bending with the twist row (no bending incompatible modes in the
    // macro quads) plus MacNeal's shear.
    for (int it = tl; it < 30; it += T3_TEAM) {
        const int q = it / 10, pp = it - 10 * q;
        int ka, kb;
        q4_pair(pp, ka, kb);
        double v[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        bend_pair(S.u.q.dNx[q], S.u.q.dNy[q], S.u.q.wdet[q], ka, kb, cb, nu, gam, v);
        if (macneal) macneal_pair(S.u.q.Dd[q], S.u.q.W[q], ka, kb, v);
        const double vf[9] = {v[0][0], v[0][1], v[0][2], v[1][0], v[1][1], v[1][2], v[2][0], v[2][1], v[2][2]};
        st9(S.Pb[q][pp], vf);
    }
    __syncwarp(tm);
}

// Condensation of the internal dofs: X = Kii^-1 Kie into S.u.c.X.
__device__ __forceinline__ void t3_condense(T3KShared &S, int tl, unsigned tm) {
    // Phase 3: lane r < 12 holds row r of [Kii | Kie] (internal dof r =
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
    double diag = 1.0;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        const bool is_piv = tl == k;  // diagonal pivot: the row of lane k
        const double akk = __shfl_sync(tm, row[k], k, 16);
        if (is_piv) diag = akk;
        const double f = (act && !is_piv) ? row[k] / akk : 0.0;
#pragma unroll
        for (int j = k + 1; j < 21; ++j) {
            const double pj = __shfl_sync(tm, row[j], k, 16);
            row[j] -= f * pj;
        }
    }
    __syncwarp(tm);  // every lane is past its last read of the quad data
    if (act)
#pragma unroll
        for (int c = 0; c < 9; ++c) S.u.c.X[tl][c] = row[12 + c] / diag;
    __syncwarp(tm);
}

// Blocks of the 7-node macro system: nodes ordered midpoints 3, 4, 5,
// centroid 6, corners 0, 1, 2; block (I, J), I <= J, packed upper-triangular.
__host__ __device__ constexpr int t3_pblk(int I, int J) { return I * 7 - I * (I - 1) / 2 + (J - I); }
__host__ __device__ constexpr int t3_mnode(int I) { return I < 4 ? I + 3 : I - 4; }

// Macro blocks of the stiffness kernel, summed where they are computed.
// Each of the 30 (virtual quad, node pair) plate blocks belongs to one upper
// block (I, J) of the macro system (transposed when the quad's pair runs
// against the node order), and every block's contributions sit on one lane
// in quad order, so block I J is ((P_q0 + P_q1) + P_q2) as a sum over the
// quads would give.  Entry [round][lane]: quad (bits 0-1), local pair (2-5),
// block (6-10), transpose (11), mode (12-13): store, add to the block, store
// to the spare block (the centroid's third quad, added by t3_schur), none.
// Lanes 0-5 take the six blocks with two quads, lanes 6-7 the centroid's
// three, lanes 7-14 the fifteen blocks with one; lane 15 zeroes the blocks
// no quad touches that the elimination reads (its first step skips corner 2,
// which shares no quad with midpoint 3).
__device__ const uint16_t c_t3_macro_items[2][16] = {
    {0x0010, 0x00d4, 0x01d1, 0x0255, 0x0364, 0x0ba0, 0x049c, 0x249e, 0x0098, 0x094d, 0x0ac5, 0x0bcc, 0x0cc8, 0x0d4a, 0x0641, 0x3000},
    {0x1025, 0x18e1, 0x11e6, 0x1a62, 0x1352, 0x1396, 0x149d, 0x0859, 0x0904, 0x0a1a, 0x0b0e, 0x0c46, 0x0d09, 0x0580, 0x06c2, 0x3000},
};
constexpr int T3_SPARE_BLOCK = 28;  // the centroid block's third contribution

__device__ __forceinline__ void t3_macro_blocks(T3KShared &S, double (*A)[10], int tl, unsigned tm, double cb, double nu,
                                                double gam, bool macneal) {
    const int code[2] = {__ldg(&c_t3_macro_items[0][tl]), __ldg(&c_t3_macro_items[1][tl])};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int c = code[r], mode = c >> 12;
        if (mode == 3) continue;
        const int q = c & 3, pp = (c >> 2) & 15, b = (c >> 6) & 31;
        const bool tr = (c >> 11) & 1;
        int ka, kb;
        q4_pair(pp, ka, kb);
        double v[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        bend_pair(S.u.q.dNx[q], S.u.q.dNy[q], S.u.q.wdet[q], ka, kb, cb, nu, gam, v);
        if (macneal) macneal_pair(S.u.q.Dd[q], S.u.q.W[q], ka, kb, v);
        double f[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) f[3 * i + j] = tr ? v[j][i] : v[i][j];
        double *dst = A[mode == 2 ? T3_SPARE_BLOCK : b];
        if (mode == 1) {
            double o[9];
            ld9(dst, o);
#pragma unroll
            for (int i = 0; i < 9; ++i) f[i] = o[i] + f[i];
        }
        st9(dst, f);
    }
    if (tl == 15) {
        const double z[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        st9(A[t3_pblk(1, 4)], z); st9(A[t3_pblk(2, 5)], z);
        st9(A[t3_pblk(4, 5)], z); st9(A[t3_pblk(4, 6)], z); st9(A[t3_pblk(5, 6)], z);
    }
    __syncwarp(tm);
}

// Condensed plate stiffness Kc = Kee - Kei Kii^-1 Kie, for the stiffness
// kernel, by 3x3-block elimination of the four internal nodes from the macro
// blocks of t3_macro_blocks.  For each internal node K: its pivot block
// D = L diag(d) L' in closed form (1/D00, D00/m2 and m2/det from one
// reciprocal of D00 m2 det), Z_J = L^-1 A_KJ and Zs_J = diag(d)^-1 Z_J for
// every later node J, and every later block A_IJ -= Z_I' Zs_J.  Kii is
// symmetric positive definite, so this unpivoted elimination matches the
// reference's pivoted LU up to rounding.  On return the corner blocks
// (4 + a, 4 + b) of A hold Kc.  Lanes 12-14, idle in the first step, form the
// corners' node blocks S.Qn for the write phase (T R_k with CD frames, else T).
__device__ __forceinline__ void t3_schur(T3KShared &S, double (*A)[10], int tl, unsigned tm, bool frames) {
    double *Zb = &S.u.z.Z[0][0];  // step K, later node J = K + 1 + j: Z at 20 j, Zs at 20 j + 10
#pragma unroll
    for (int K = 0; K < 4; ++K) {
        // the first step's last node, corner 2, has a zero block with midpoint 3 (no shared quad):
        // its Z and every update through it are zero and skipped
        const int n = K == 0 ? 5 : 6 - K;
        double D[9];
        ld9(A[t3_pblk(K, K)], D);
        const double D00 = D[0], D01 = D[1], D02 = D[2], D11 = D[4], D12 = D[5], D22 = D[8];
        const double m2 = D00 * D11 - D01 * D01;
        const double det = D00 * (D11 * D22 - D12 * D12) - D01 * (D01 * D22 - D12 * D02) + D02 * (D01 * D12 - D11 * D02);
        // 1/D00, D00/m2 and m2/det from one reciprocal of D00 m2 det
        const double r = 1.0 / (D00 * m2 * det);
        const double i0 = (m2 * det) * r, i1 = D00 * ((D00 * det) * r), i2 = m2 * ((D00 * m2) * r);
        const double l10 = D01 * i0, l20 = D02 * i0, l21 = (D12 - l20 * D01) * i1;
        if (tl < n) {
            double B[9], z[9], zs[9];
            ld9(A[t3_pblk(K, K + 1 + tl)], B);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double z0 = B[c], z1 = B[3 + c] - l10 * z0, z2 = B[6 + c] - l20 * z0 - l21 * z1;
                z[c] = z0; z[3 + c] = z1; z[6 + c] = z2;
                zs[c] = z0 * i0; zs[3 + c] = z1 * i1; zs[6 + c] = z2 * i2;
            }
            st9(Zb + 20 * tl, z);
            st9(Zb + 20 * tl + 10, zs);
        } else if (K == 0 && tl == 15) {
            // the centroid block's third quad, before the first update reads the block
            double c3[9], s3[9];
            ld9(A[t3_pblk(3, 3)], c3);
            ld9(A[T3_SPARE_BLOCK], s3);
#pragma unroll
            for (int i = 0; i < 9; ++i) c3[i] = c3[i] + s3[i];
            st9(A[t3_pblk(3, 3)], c3);
        } else if (K == 0 && tl >= 12) {
            const int k = tl - 12;
            double Q[9];
            if (frames) {
                node_block(S.V, S.V + 3, S.V + 6, S.R[k], Q);
            } else {
#pragma unroll
                for (int i = 0; i < 9; ++i) Q[i] = S.V[i];
            }
            st9(S.Qn[k], Q);
        }
        __syncwarp(tm);
        for (int t = tl; t < n * (n + 1) / 2; t += T3_TEAM) {
            int ip = 0, rem = t;
            while (rem >= n - ip) { rem -= n - ip; ++ip; }
            const int jp = ip + rem;
            double Zi[9], Zs[9], C[9];
            ld9(Zb + 20 * ip, Zi);
            ld9(Zb + 20 * jp + 10, Zs);
            double *Cp = A[t3_pblk(K + 1 + ip, K + 1 + jp)];
            ld9(Cp, C);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    C[3 * r + c] -= Zi[r] * Zs[c] + Zi[3 + r] * Zs[3 + c] + Zi[6 + r] * Zs[6 + c];
            st9(Cp, C);
        }
        __syncwarp(tm);
    }
}

// Sub-block (bi, bj) of a node-pair 6x6 block into a staged slot buffer of
// 36 values in stored orientation (transposed when the slot says so).
__device__ __forceinline__ void stage_sub_block(double *buf, bool t, int bi, int bj, const double O[3][3], double &lmax) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double v = O[i][j];
            lmax = fmax(lmax, fabs(v));
            const int r = 3 * bi + i, c = 3 * bj + j;
            buf[t ? 6 * c + r : 6 * r + c] = v;
        }
}

// W warps per CTA (2 W elements): 2 or 4, both at 20 warps per SM.
template <int W>
__global__ void __launch_bounds__(32 * W, W == 2 ? 10 : 5) t3_k_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                         const double *__restrict__ prop,
                                                         const double *__restrict__ coords,
                                                         const double *__restrict__ nodeR, double k6rot, ElemOut o) {
    __shared__ T3KShared sh[T3_TEAMS_PER_WARP * W];
    o = o.at(blockIdx.y);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane >> 4, tl = lane & 15;
    const unsigned tm = 0xFFFFu << (16 * team);
    const int64_t e = (int64_t)blockIdx.x * (T3_TEAMS_PER_WARP * W) + warp * T3_TEAMS_PER_WARP + team;
    if (e >= nt) return;  // the whole team leaves; syncs below are team-local
    T3KShared &S = sh[warp * T3_TEAMS_PER_WARP + team];
    // lane tl < 12's node-pair slot (pair tl / 2), loaded now so that its latency hides behind the element's work
    const int32_t sl_early = tl < 12 ? __ldg(o.blk_slot + e * 6 + (tl >> 1)) : -1;

    // Phase 0, every lane in registers: nodes, corners, properties, frame,
    // local coordinates, CST derivatives, constitutive scalars.
    double x[3], y[3], A, cb, cs, nu, gam;
    bool plate, macneal;
    {
        const double *pr = prop + 7 * e;
        const double h = o.thickness(e, pr), E = __ldg(pr + 1), br = __ldg(pr + 4), tst = __ldg(pr + 5), Gs = __ldg(pr + 6);
        nu = __ldg(pr + 2);
        int nd[3];
        double p[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            nd[k] = __ldg(nodes + 3 * e + k);
#pragma unroll
            for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
        }
        // the corners' CD frames into shared memory now, off the output phase's path
        if (nodeR)
            for (int i = tl; i < 27; i += T3_TEAM) {
                const int k = i < 9 ? 0 : (i < 18 ? 1 : 2);
                const int64_t n = k == 0 ? nd[0] : (k == 1 ? nd[1] : nd[2]);
                S.R[k][i - 9 * k] = __ldg(nodeR + 9 * n + (i - 9 * k));
            }
        double v1[3], v2[3], v3[3];
        t3_frame(p[0], p[1], p[2], v1, v2, v3);
        double c[3];
        for (int i = 0; i < 3; ++i) c[i] = (p[0][i] + p[1][i] + p[2][i]) * (1.0 / 3.0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double d[3];
            sub3(p[k], c, d);
            x[k] = dot3(d, v1);
            y[k] = dot3(d, v2);
        }
        A = 0.5 * fabs(x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]));
        gam = (1 - nu) / 2;
        const double inu = 1.0 / (1 - nu * nu);  // one reciprocal for cm and cb
        const double cm = E * h * inu;
        cb = br * (E * h * h * h) * (inu * (1.0 / 12.0));
        const bool membrane_only = br <= 1e-12;
        cs = membrane_only ? 0.0 : tst * h * Gs;
        plate = !membrane_only && A >= 1e-12;
        macneal = plate && !(h < 1e-30 || fabs(cs) < 1e-30);
        if (tl == 0) {
            for (int i = 0; i < 3; ++i) { S.V[i] = v1[i]; S.V[3 + i] = v2[i]; S.V[6 + i] = v3[i]; S.nd[i] = nd[i]; }
            const double i2A = 1.0 / (2 * A);
            S.bv[0] = (y[1] - y[2]) * i2A; S.bv[1] = (y[2] - y[0]) * i2A; S.bv[2] = (y[0] - y[1]) * i2A;
            S.cv[0] = (x[2] - x[1]) * i2A; S.cv[1] = (x[0] - x[2]) * i2A; S.cv[2] = (x[1] - x[0]) * i2A;
            S.A = A;
            S.cm = cm;
            // G_ref = shear-material G (assembly.jl:2468)
            S.ad = ((membrane_only ? 0.0 : k6rot) / 1e5) * Gs * h;
        }
    }

    double(*Am)[10] = reinterpret_cast<double(*)[10]>(&S.Pb[0][0][0]);  // the macro blocks
    if (plate) {
        t3_plate_points(S, tl, tm, x, y, cs, cb, macneal);
        // Phases 2-4: macro blocks, then Kcond = Kee - Kei Kii^-1 Kie by
        // 3x3-block elimination (Kee and Kei from the corner's own quad)
        t3_macro_blocks(S, Am, tl, tm, cb, nu, gam, macneal);
        t3_schur(S, Am, tl, tm, nodeR != nullptr);
    }
    __syncwarp(tm);

    // Phase 5: lane tl < 12 takes node pair tl / 2 and sub-block row bi =
    // tl % 2 (translations, rotations) for both sub-block columns.  Local
    // block: CST membrane and centroidal drill on (u, v, theta_z), condensed
    // plate on (w, theta_x, theta_y).
    double lmax = 0.0;
    if (tl < 12) {
        const int pair = tl >> 1, bi = tl & 1;
        const int a = (pair >= 3) + (pair >= 5);
        const int b = a + pair - (a == 0 ? 0 : (a == 1 ? 3 : 5));
        double Lm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Lp[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (A >= 1e-12) {
            const double ba = S.bv[a], ca = S.cv[a], bb = S.bv[b], cb_ = S.cv[b], cm = S.cm, ad = S.ad;
            const double da[3] = {0.5 * ca, -0.5 * ba, 1.0 / 3.0}, db[3] = {0.5 * cb_, -0.5 * bb, 1.0 / 3.0};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) Lm[i][j] = ad * (da[i] * db[j]) * A;
            Lm[0][0] += (cm * (ba * bb + gam * (ca * cb_))) * A;
            Lm[0][1] += (cm * (nu * (ba * cb_) + gam * (ca * bb))) * A;
            Lm[1][0] += (cm * (nu * (ca * bb) + gam * (ba * cb_))) * A;
            Lm[1][1] += (cm * (ca * cb_ + gam * (ba * bb))) * A;
            if (plate) {
                double kc[9];
                ld9(Am[t3_pblk(4 + a, 4 + b)], kc);
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) Lp[i][j] = kc[3 * i + j];
            }
        }
        double Qa[9], Qb[9];
        if (plate) {  // formed during the block elimination
            ld9(S.Qn[a], Qa);
            ld9(S.Qn[b], Qb);
        } else if (nodeR) {
            node_block(S.V, S.V + 3, S.V + 6, S.R[a], Qa);
            node_block(S.V, S.V + 3, S.V + 6, S.R[b], Qb);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) { Qa[i] = S.V[i]; Qb[i] = S.V[i]; }
        }
        const int32_t sl = sl_early;
        // Regular slots are staged in S.u.o (free after phase 4) in their
        // stored orientation and copied out below as bulk copies; pairs on the
        // RBE2 path are written directly.
        double *buf = S.u.o.O[pair];
        const bool t = sl >= 0 && (sl & kBlkTranspose);
        double M[3][3], O[3][3];
        // diagonal sub-block: (u, v, w) x (u, v, w) or (rx, ry, rz) x (rx, ry, rz)
        M[0][0] = bi ? Lp[1][1] : Lm[0][0]; M[0][1] = bi ? Lp[1][2] : Lm[0][1];
        M[1][0] = bi ? Lp[2][1] : Lm[1][0]; M[1][1] = bi ? Lp[2][2] : Lm[1][1];
        M[2][2] = bi ? Lm[2][2] : Lp[0][0];
        rot_sparse<0b100011011>(Qa, M, Qb, O);
        if (sl < 0) {
            write_sub_block(o, e, sl, a, b, bi, bi, O, lmax, 18);
        } else {
            stage_sub_block(buf, t, bi, bi, O, lmax);
            if (o.diag_staging && a == b)
#pragma unroll
                for (int i = 0; i < 3; ++i) o.diag_staging[__ldg(o.diag_slot + e * 18 + 6 * a + 3 * bi + i)] = O[i][i];
        }
        // off-diagonal sub-block: (u, v, w) x (rx, ry, rz) or its mirror
        M[0][2] = bi ? Lp[1][0] : Lm[0][2]; M[1][2] = bi ? Lp[2][0] : Lm[1][2];
        M[2][0] = bi ? Lm[2][0] : Lp[0][1]; M[2][1] = bi ? Lm[2][1] : Lp[0][2];
        rot_sparse<0b011100100>(Qa, M, Qb, O);
        if (sl < 0) write_sub_block(o, e, sl, a, b, bi, 1 - bi, O, lmax, 18);
        else stage_sub_block(buf, t, bi, 1 - bi, O, lmax);
        if (bi == 0) S.slot[pair] = sl;
    }
    slot_fence();  // the staged values, written by two lanes per slot, before the bulk copies
    __syncwarp(tm);
    // lane p < 6 copies staged slot p out as one 288-byte bulk copy
    if (tl < 6) {
        const int32_t st = S.slot[tl];
        if (st >= 0) slot_copy(o.staging + 36 * (int64_t)(st & kBlkIndexMask), S.u.o.O[tl], 288);
    }
    if (o.maxabs) {
        for (int off = 8; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(tm, lmax, off, 16));
        if (tl == 0 && lmax > 0.0) atomic_max_nonneg(o.maxabs, lmax);
    }
    slot_copies_read();
}

// One CTRIA3 per thread: frame, node blocks and the CST membrane stress
// once, then the six node-pair blocks s_ab * Q_a' Q_b (shell KG acts on
// translations only).
// Dynamic shared memory: T3KG_STAGE_STRIDE doubles per thread, two staged
// slots of 12 that alternate as the slots leave by bulk copies (a buffer is
// refilled once the copy issued before the latest one has read it).  The
// 26-double stride puts a warp's 16-byte stores on all eight bank groups.
constexpr int T3KG_STAGE_STRIDE = 26;
__global__ void __launch_bounds__(128) t3_kg_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                   const double *__restrict__ prop,
                                                   const double *__restrict__ coords,
                                                   const double *__restrict__ nodeR,
                                                   const double *__restrict__ u, ElemOut o) {
    extern __shared__ __align__(16) double t3kg_smem[];
    double *sbuf = t3kg_smem + T3KG_STAGE_STRIDE * threadIdx.x;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nt) return;
    o = o.at(blockIdx.y);
    u += (int64_t)blockIdx.y * o.u_stride;
    int32_t nd[3];
    double p[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        nd[k] = __ldg(nodes + 3 * e + k);
#pragma unroll
        for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
    }
    double v1[3], v2[3], v3[3];
    t3_frame(p[0], p[1], p[2], v1, v2, v3);
    double c[3], lc[3][2];
#pragma unroll
    for (int i = 0; i < 3; ++i) c[i] = (p[0][i] + p[1][i] + p[2][i]) * (1.0 / 3.0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double d[3];
        sub3(p[k], c, d);
        lc[k][0] = dot3(d, v1);
        lc[k][1] = dot3(d, v2);
    }
    double Q[3][9];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double Rl[9];
        if (nodeR)
#pragma unroll
            for (int i = 0; i < 9; ++i) Rl[i] = __ldg(nodeR + 9 * (int64_t)nd[k] + i);
        node_block(v1, v2, v3, nodeR ? Rl : nullptr, Q[k]);
    }
    const double *pr = prop + 7 * e;
    const double h = o.thickness(e, pr), E = __ldg(pr + 1), nu = __ldg(pr + 2);
    const double x[3] = {lc[0][0], lc[1][0], lc[2][0]}, y[3] = {lc[0][1], lc[1][1], lc[2][1]};
    const double A = 0.5 * fabs(x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]));
    double val[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (A >= 1e-12 && h >= 1e-30) {
        const double b[3] = {(y[1] - y[2]) / (2 * A), (y[2] - y[0]) / (2 * A), (y[0] - y[1]) / (2 * A)};
        const double cv[3] = {(x[2] - x[1]) / (2 * A), (x[0] - x[2]) / (2 * A), (x[1] - x[0]) / (2 * A)};
        double eps0 = 0.0, eps1 = 0.0, eps2 = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double *ug = u + 6 * (int64_t)nd[k];
            const double u0 = __ldg(ug), u1 = __ldg(ug + 1), u2 = __ldg(ug + 2);
            const double ul = Q[k][0] * u0 + Q[k][1] * u1 + Q[k][2] * u2;
            const double vl = Q[k][3] * u0 + Q[k][4] * u1 + Q[k][5] * u2;
            eps0 += b[k] * ul;
            eps1 += cv[k] * vl;
            eps2 += cv[k] * ul + b[k] * vl;
        }
        const double cm = E / (1 - nu * nu);
        const double Nx = (cm * eps0 + cm * nu * eps1) * h;
        const double Ny = (cm * nu * eps0 + cm * eps1) * h;
        const double Nxy = (cm * (1 - nu) / 2 * eps2) * h;
        const double sxx = Nx / h, syy = Ny / h, sxy = Nxy / h;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                val[i][j] = h * A * (sxx * b[i] * b[j] + syy * cv[i] * cv[j] + sxy * (b[i] * cv[j] + cv[i] * b[j]));
    }
    int ncopy = 0;
#pragma unroll
    for (int pp = 0; pp < 6; ++pp) {
        const int pa = (pp >= 3) + (pp >= 5), pb = pa + pp - (pa == 0 ? 0 : (pa == 1 ? 3 : 5));
        const double L[3][3] = {{val[pa][pb], 0, 0}, {0, val[pa][pb], 0}, {0, 0, val[pa][pb]}};
        double O[3][3];
        rot_block(Q[pa], L, Q[pb], O);
        const int32_t sl = __ldg(o.blk_slot + e * 6 + pp);
        if (sl >= 0) {
            // staged blocks of KG shells are read as their translation 3x3 only:
            // the 3x3 in stored orientation and three zeros, one 96-byte copy
            const bool t = sl & kBlkTranspose;
            double *sb = sbuf + 12 * (ncopy & 1);
            if (ncopy >= 2) slot_copies_read_but_last();
            double2 *s2 = reinterpret_cast<double2 *>(sb);
            const double v0 = O[0][0], v1 = t ? O[1][0] : O[0][1], v2 = t ? O[2][0] : O[0][2];
            const double v3 = t ? O[0][1] : O[1][0], v4 = O[1][1], v5 = t ? O[2][1] : O[1][2];
            const double v6 = t ? O[0][2] : O[2][0], v7 = t ? O[1][2] : O[2][1], v8 = O[2][2];
            s2[0] = make_double2(v0, v1); s2[1] = make_double2(v2, v3); s2[2] = make_double2(v4, v5);
            s2[3] = make_double2(v6, v7); s2[4] = make_double2(v8, 0.0); s2[5] = make_double2(0.0, 0.0);
            slot_fence();
            slot_copy(o.staging + 12 * (int64_t)(sl & kBlkIndexMask), sb, 96);
            ++ncopy;
        } else {
            // the dof-level RBE2 path reads whole raw blocks
#pragma unroll
            for (int i = 0; i < 6; ++i)
#pragma unroll
                for (int j = 0; j < 6; ++j) *blk_entry(o, sl, i, j) = (i < 3 && j < 3) ? O[i][j] : 0.0;
        }
    }
    slot_copies_read();
}

}  // namespace jfg
