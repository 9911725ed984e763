// elem_recover.cuh -- SOL 101 output recovery: shell forces, moments, shears,
// fibre stresses and strains, CQUAD4 bilinear corner forces, and CBAR/CBEAM
// end forces and section stresses (recover_shell_stresses! and
// recover_bar_stresses!, src/solver/stress_recovery.jl:163-593, default
// branch: isotropic PSHELL/MAT1, no SNORM, no curvature membrane).
//
// CQUAD4: one thread per element.  stress_strain_quad4 and
// quad4_bilinear_corner_forces (src/FEMKernels.jl:6003-6338) share their two
// Gauss loops, so the thread runs them once: the Wilson-mode amplitudes
// alpha = -(K_bb \ K_ab' u) come from Gauss-point membrane stresses
// (K_ab' u = sum_g |J_g| Bi_g' Cm Bm_g u, no 24x4 matrix), then the strains
// at the Gauss points give the area averages and the corner extrapolation.
// CTRIA3: a team of 16 lanes reuses the stiffness kernel's plate phases with
// the recovery constitutive set (Cb = D h^3/12, Cs = 5/6 G h), condenses the
// virtual-quad macro, and three lanes recover one virtual quad each.
// CBAR/CBEAM: one thread per bar, k u in the bar frame with compile-time
// frame-matrix entries.
#pragma once
#include "elem_bar.cuh"
#include "elem_t3.cuh"

namespace jfg {

constexpr int REC_SHELL = 48;  // JFG_SHELL_REC
constexpr int REC_BAR = 18;    // JFG_BAR_REC

// y = D x for the plane-stress D = c [1 nu 0; nu 1 0; 0 0 (1 - nu)/2].
__device__ __forceinline__ void ps_mul(double c, double nu, const double x[3], double y[3]) {
    const double cn = c * nu, cg = c * ((1 - nu) / 2);
    y[0] = c * x[0] + cn * x[1];
    y[1] = cn * x[0] + c * x[1];
    y[2] = cg * x[2];
}

// Local displacements of a shell node: T_k u_k with T_k = Rel * node_R.
__device__ __forceinline__ void shell_node_local(const double V[9], const double *__restrict__ nodeR, int32_t nd,
                                                 const double *__restrict__ u, double ul[6]) {
    double Q[9];
    if (nodeR) {
        double R[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) R[i] = __ldg(nodeR + 9 * (int64_t)nd + i);
        node_block(V, V + 3, V + 6, R, Q);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) Q[i] = V[i];
    }
    double ug[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) ug[i] = __ldg(u + 6 * (int64_t)nd + i);
#pragma unroll
    for (int half = 0; half < 2; ++half)
#pragma unroll
        for (int r = 0; r < 3; ++r)
            ul[3 * half + r] = Q[3 * r] * ug[3 * half] + Q[3 * r + 1] * ug[3 * half + 1] + Q[3 * r + 2] * ug[3 * half + 2];
}

// quad4_mitc4_center_shear_resultant (FEMKernels.jl:5927-6001): covariant
// shear from the four tying points, centre Jacobian, PHI2_ALPHA = 10, ts_t 5/6.
// w, tx, ty: the corners' plate dofs (w, theta_x, theta_y).
__device__ __forceinline__ void mitc4_center_shear(const double lc[4][2], const double w[4], const double tx[4],
                                                   const double ty[4], double G, double h, double Q[2]) {
    double g0 = 0.0, g1 = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const double xi = t == 2 ? -1.0 : (t == 3 ? 1.0 : 0.0), eta = t == 0 ? -1.0 : (t == 1 ? 1.0 : 0.0);
        const double dNr[4] = {-0.25 * (1 - eta), 0.25 * (1 - eta), 0.25 * (1 + eta), -0.25 * (1 + eta)};
        const double dNs[4] = {-0.25 * (1 - xi), -0.25 * (1 + xi), 0.25 * (1 + xi), 0.25 * (1 - xi)};
        const double Nt[4] = {0.25 * (1 - xi) * (1 - eta), 0.25 * (1 + xi) * (1 - eta), 0.25 * (1 + xi) * (1 + eta),
                              0.25 * (1 - xi) * (1 + eta)};
        double Ja = 0.0, Jb = 0.0;  // (J11, J12) at the xi-direction points, (J21, J22) at the eta-direction ones
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double d = t < 2 ? dNr[k] : dNs[k];
            Ja += d * lc[k][0];
            Jb += d * lc[k][1];
        }
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) s += (t < 2 ? dNr[k] : dNs[k]) * w[k] + (-Jb * Nt[k]) * tx[k] + (Ja * Nt[k]) * ty[k];
        if (t < 2) g0 += 0.5 * s;
        else g1 += 0.5 * s;
    }
    double J11 = 0.0, J12 = 0.0, J21 = 0.0, J22 = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double dr = (k == 1 || k == 2) ? 0.25 : -0.25, ds = k >= 2 ? 0.25 : -0.25;
        J11 += dr * lc[k][0]; J12 += dr * lc[k][1];
        J21 += ds * lc[k][0]; J22 += ds * lc[k][1];
    }
    const double det = J11 * J22 - J12 * J21;
    const double adet = fmax(fabs(det), 1e-30), inv = 1.0 / det;
    const double i11 = J22 * inv, i12 = -J12 * inv, i21 = -J21 * inv, i22 = J11 * inv;
    const double phi2 = fmin(1.0, 10.0 * h * h / fmax(4.0 * adet, 1e-30));
    const double k = 5.0 / 6.0 * G * h;
    const double t11 = k * i11, t12 = k * i12, t21 = k * i21, t22 = k * i22;
    const double q1 = phi2 * ((i11 * t11 + i21 * t21) * g0 + (i11 * t12 + i21 * t22) * g1);
    const double q2 = phi2 * ((i12 * t11 + i22 * t21) * g0 + (i12 * t12 + i22 * t22) * g1);
    Q[0] = J11 * q1 + J21 * q2;
    Q[1] = J12 * q1 + J22 * q2;
}

// Principal stress (compute_principal_2d, FEMKernels.jl:5921-5925, first
// root) and von Mises of a membrane stress triple.
__device__ __forceinline__ double principal_max(const double s[3]) {
    const double hd = (s[0] - s[1]) / 2.0;
    return (s[0] + s[1]) / 2.0 + sqrt(hd * hd + s[2] * s[2]);
}
__device__ __forceinline__ double von_mises(const double s[3]) {
    return sqrt(s[0] * s[0] - s[0] * s[1] + s[1] * s[1] + 3 * s[2] * s[2]);
}

// The shell record's common part (forces, fibre stresses and strains).
__device__ __forceinline__ void put_shell_rec(double *o, const double N[3], const double M[3], const double Q[2],
                                              const double ez1[3], const double ez2[3], double c, double nu) {
    double sz1[3], sz2[3];
    ps_mul(c, nu, ez1, sz1);
    ps_mul(c, nu, ez2, sz2);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o[k] = N[k]; o[3 + k] = M[k];
        o[8 + k] = sz1[k]; o[11 + k] = sz2[k]; o[14 + k] = ez1[k]; o[17 + k] = ez2[k];
    }
    o[6] = Q[0]; o[7] = Q[1];
    o[20] = principal_max(sz1);
    o[21] = 1.0;
    o[46] = von_mises(sz1);
    o[47] = von_mises(sz2);
}

// 4x4 solve with partial pivoting (the reference's K_bb \ rhs); false on an
// exactly zero pivot.
__device__ __forceinline__ bool solve4(double A[4][4], double b[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int p = k;
        double best = fabs(A[k][k]);
#pragma unroll
        for (int i = k + 1; i < 4; ++i)
            if (fabs(A[i][k]) > best) { best = fabs(A[i][k]); p = i; }
        if (best == 0.0) return false;
        if (p != k) {
#pragma unroll
            for (int j = 0; j < 4; ++j) { const double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
            const double t = b[k]; b[k] = b[p]; b[p] = t;
        }
#pragma unroll
        for (int i = k + 1; i < 4; ++i) {
            const double f = A[i][k] / A[k][k];
#pragma unroll
            for (int j = k + 1; j < 4; ++j) A[i][j] -= f * A[k][j];
            b[i] -= f * b[k];
        }
    }
#pragma unroll
    for (int k = 3; k >= 0; --k) {
        double s = b[k];
#pragma unroll
        for (int i = k + 1; i < 4; ++i) s -= A[k][i] * b[i];
        b[k] = s / A[k][k];
    }
    return true;
}

// quad4_is_axis_aligned_rectangle (FEMKernels.jl:5050-5077), tol 1e-8.
__device__ __forceinline__ bool q4_is_rectangle(const double lc[4][2]) {
    const double tol = 1e-8;
    double ex[4], ey[4], L[4], Lmax = 1e-12;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int n = (k + 1) & 3;
        ex[k] = lc[n][0] - lc[k][0];
        ey[k] = lc[n][1] - lc[k][1];
        L[k] = sqrt(ex[k] * ex[k] + ey[k] * ey[k]);
        Lmax = fmax(Lmax, L[k]);
    }
    const double as = Lmax * Lmax;
    if (fabs(ex[0] * ey[2] - ey[0] * ex[2]) > tol * as || fabs(ex[1] * ey[3] - ey[1] * ex[3]) > tol * as) return false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int n = (k + 1) & 3;
        if (fabs(ex[k] * ex[n] + ey[k] * ey[n]) > tol * as) return false;
    }
    return !(fabs(L[0] - L[2]) > tol * Lmax || fabs(L[1] - L[3]) > tol * Lmax);
}

// CQUAD4 branch of recover_shell_stresses! (stress_recovery.jl:179-302):
// element e's record into o.
__device__ __forceinline__ void q4_recover_element(int64_t e, const int32_t *__restrict__ nodes,
                                                   const double *__restrict__ prop, const double *__restrict__ coords,
                                                   const double *__restrict__ nodeR, const double *__restrict__ u,
                                                   bool pressure_deck, double *o) {
    const double *pr = prop + 7 * e;
    const double h = __ldg(pr), E = __ldg(pr + 1), nu = __ldg(pr + 2), br = __ldg(pr + 4);
    int32_t nd[4];
    double p[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        nd[k] = __ldg(nodes + 4 * e + k);
#pragma unroll
        for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
    }
    double V[9], lc[4][2];
    q4_local(p, V, lc);
    double ul[4][6];
#pragma unroll
    for (int k = 0; k < 4; ++k) shell_node_local(V, nodeR, nd[k], u, ul[k]);

    const double c = E / (1 - nu * nu), cm = c * h, cb = br * c * (h * h * h / 12.0);
    double J11 = 0.0, J12 = 0.0, J21 = 0.0, J22 = 0.0;  // centre Jacobian
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double dr = (k == 1 || k == 2) ? 0.25 : -0.25, ds = k >= 2 ? 0.25 : -0.25;
        J11 += dr * lc[k][0]; J12 += dr * lc[k][1];
        J21 += ds * lc[k][0]; J22 += ds * lc[k][1];
    }
    // Gauss loop: compatible membrane strain, curvature, Wilson-mode B and
    // the condensation system
    double em[4][3], kap[4][3], bi[4][4], wd[4];  // bi: d(phi1)/dx, d(phi1)/dy, d(phi2)/dx, d(phi2)/dy
    double Kbb[4][4], rhs[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) Kbb[i][j] = 0.0;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        double r, s, dx[4], dy[4], iJ[4];
        q4_shape_gp(g, r, s);
        const double det = q4_point_derivs(lc, r, s, false, dx, dy, iJ);
        const double w = fabs(det) < 1e-12 ? 1e-12 : fabs(det);
        wd[g] = w;
        double e0 = 0, e1 = 0, e2 = 0, k0 = 0, k1 = 0, k2 = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            e0 += dx[k] * ul[k][0]; e1 += dy[k] * ul[k][1]; e2 += dy[k] * ul[k][0] + dx[k] * ul[k][1];
            k0 += dx[k] * ul[k][4]; k1 += -dy[k] * ul[k][3]; k2 += dy[k] * ul[k][4] - dx[k] * ul[k][3];
        }
        em[g][0] = e0; em[g][1] = e1; em[g][2] = e2;
        kap[g][0] = k0; kap[g][1] = k1; kap[g][2] = k2;
        bi[g][0] = iJ[0] * (-2.0 * r); bi[g][1] = iJ[2] * (-2.0 * r);
        bi[g][2] = iJ[1] * (-2.0 * s); bi[g][3] = iJ[3] * (-2.0 * s);
        // columns of Bi: (d1x, 0, d1y), (0, d1y, d1x), (d2x, 0, d2y), (0, d2y, d2x)
        double col[4][3] = {{bi[g][0], 0.0, bi[g][1]}, {0.0, bi[g][1], bi[g][0]},
                            {bi[g][2], 0.0, bi[g][3]}, {0.0, bi[g][3], bi[g][2]}};
        double sig[3];
        ps_mul(cm, nu, em[g], sig);
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            rhs[l] += w * (sig[0] * col[l][0] + sig[1] * col[l][1] + sig[2] * col[l][2]);
            double cc[3];
            ps_mul(cm, nu, col[l], cc);
#pragma unroll
            for (int mm = 0; mm < 4; ++mm) Kbb[mm][l] += w * (col[mm][0] * cc[0] + col[mm][1] * cc[1] + col[mm][2] * cc[2]);
        }
    }
    const bool ok = J11 * J22 - J12 * J21 != 0.0 && solve4(Kbb, rhs);
    if (!ok) {
        // the reference's try block fails (singular centre Jacobian or K_bb): no output
        for (int i = 0; i < REC_SHELL; ++i) o[i] = 0.0;
        return;
    }
    // strains with the incompatible modes (alpha = -rhs), area averages
    double ea[3] = {0, 0, 0}, ka[3] = {0, 0, 0}, area = 0.0;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        em[g][0] += bi[g][0] * (-rhs[0]) + bi[g][2] * (-rhs[2]);
        em[g][1] += bi[g][1] * (-rhs[1]) + bi[g][3] * (-rhs[3]);
        em[g][2] += bi[g][1] * (-rhs[0]) + bi[g][0] * (-rhs[1]) + bi[g][3] * (-rhs[2]) + bi[g][2] * (-rhs[3]);
#pragma unroll
        for (int k = 0; k < 3; ++k) { ea[k] += em[g][k] * wd[g]; ka[k] += kap[g][k] * wd[g]; }
        area += wd[g];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) { ea[k] /= area; ka[k] /= area; }
    double N[3], M[3], Q[2] = {0.0, 0.0}, t[3];
    ps_mul(cm, nu, ea, N);
    ps_mul(c, nu, ka, t);
#pragma unroll
    for (int k = 0; k < 3; ++k) M[k] = -br * t[k] * (h * h * h / 12.0);
    if (br > 1e-12) {
        const double w[4] = {ul[0][2], ul[1][2], ul[2][2], ul[3][2]};
        const double tx[4] = {ul[0][3], ul[1][3], ul[2][3], ul[3][3]};
        const double ty[4] = {ul[0][4], ul[1][4], ul[2][4], ul[3][4]};
        mitc4_center_shear(lc, w, tx, ty, E / (2 * (1 + nu)), h, Q);
    }
    // bilinear corner forces: Gauss values extrapolated (interp_2x2_gauss_sigma)
    double Nc[4][3], Mc[4][3];
    {
        double Ng[4][3], Mg[4][3];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            ps_mul(cm, nu, em[g], Ng[g]);
            double mk[3];
            ps_mul(cb, nu, kap[g], mk);
#pragma unroll
            for (int k = 0; k < 3; ++k) Mg[g][k] = -mk[k];
        }
        const double pt = 0.57735026918962576451;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double xi = (i == 1 || i == 2) ? 1.0 : -1.0, eta = i >= 2 ? 1.0 : -1.0;
            const double lx1 = (pt - xi) / (2.0 * pt), lx2 = (xi + pt) / (2.0 * pt);
            const double ly1 = (pt - eta) / (2.0 * pt), ly2 = (eta + pt) / (2.0 * pt);
            const double w0 = lx1 * ly1, w1 = lx2 * ly1, w2 = lx2 * ly2, w3 = lx1 * ly2;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                Nc[i][k] = w0 * Ng[0][k] + w1 * Ng[1][k] + w2 * Ng[2][k] + w3 * Ng[3][k];
                Mc[i][k] = w0 * Mg[0][k] + w1 * Mg[1][k] + w2 * Mg[2][k] + w3 * Mg[3][k];
            }
        }
    }
    // equilibrium shear from the corner moments, kept where smaller
    // (stress_recovery.jl:88-130)
    if (fabs(br) > 1e-12) {
        const double det = J11 * J22 - J12 * J21;
        if (!(fabs(det) < 1e-12)) {
            const double i11 = J22 / det, i12 = -J12 / det, i21 = -J21 / det, i22 = J11 / det;
            double rx = 0, sx = 0, ry = 0, sy = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double dr = (k == 1 || k == 2) ? 0.25 : -0.25, ds = k >= 2 ? 0.25 : -0.25;
                rx += dr * Mc[k][0]; sx += ds * Mc[k][0]; ry += dr * Mc[k][1]; sy += ds * Mc[k][1];
            }
            const double eq0 = i11 * rx + i12 * sx, eq1 = i21 * ry + i22 * sy;
            if (isfinite(eq0) && fabs(eq0) < fabs(Q[0])) Q[0] = eq0;
            if (isfinite(eq1) && fabs(eq1) < fabs(Q[1])) Q[1] = eq1;
        }
    }
    // fibre strains use the unscaled field
    double ez1[3], ez2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { ez1[k] = ea[k] + (-h / 2.0) * ka[k]; ez2[k] = ea[k] + (h / 2.0) * ka[k]; }
    // pressure-loaded rectangle moment scale (stress_recovery.jl:131-161)
    if (pressure_deck && fabs(br) > 1e-12 && q4_is_rectangle(lc)) {
        const double mq = fmax(fabs(Q[0]), fabs(Q[1]));
        const double mn = fmax(fabs(N[0]), fmax(fabs(N[1]), fabs(N[2])));
        if (mq > 1e-8 && !(mn > fmax(1e-6, 1e-4 * mq))) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                M[k] *= 0.99;
#pragma unroll
                for (int i = 0; i < 4; ++i) Mc[i][k] *= 0.99;
            }
        }
    }
    put_shell_rec(o, N, M, Q, ez1, ez2, c, nu);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        Mc[i][2] = M[2];
#pragma unroll
        for (int k = 0; k < 3; ++k) { o[22 + 3 * i + k] = Nc[i][k]; o[34 + 3 * i + k] = Mc[i][k]; }
    }
}

// One thread per CQUAD4.  Records are built in shared memory (a row of 50
// doubles per thread, 16-byte aligned) and the block writes its contiguous
// records out as 16-byte stores; 8-byte stores when out is not 16-byte aligned.
constexpr int Q4R_THREADS = 64, Q4R_ROW = 50;
__global__ void __launch_bounds__(Q4R_THREADS) q4_recover_kernel(int64_t nq, const int32_t *__restrict__ nodes,
                                                                 const double *__restrict__ prop,
                                                                 const double *__restrict__ coords,
                                                                 const double *__restrict__ nodeR,
                                                                 const double *__restrict__ u, bool pressure_deck,
                                                                 double *__restrict__ out) {
    __shared__ __align__(16) double rec[Q4R_THREADS][Q4R_ROW];
    const int64_t e0 = (int64_t)blockIdx.x * Q4R_THREADS;
    const int t = threadIdx.x;
    if (e0 + t < nq) q4_recover_element(e0 + t, nodes, prop, coords, nodeR, u, pressure_deck, rec[t]);
    __syncthreads();
    const int n = (int)(nq - e0 < Q4R_THREADS ? nq - e0 : Q4R_THREADS);
    double *dst = out + REC_SHELL * e0;
    if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        // chunk c = 24 record + part; threads step by 64 = 2 records + 16 parts
        for (int j = t / 24, part = t % 24; j < n;) {
            reinterpret_cast<double2 *>(dst + REC_SHELL * j)[part] = reinterpret_cast<const double2 *>(rec[j])[part];
            part += 16;
            j += 2;
            if (part >= 24) { part -= 24; ++j; }
        }
    } else {
        for (int c = t; c < n * REC_SHELL; c += Q4R_THREADS) dst[c] = rec[c / REC_SHELL][c % REC_SHELL];
    }
}

// CTRIA3 branch of recover_shell_stresses! (stress_recovery.jl:303-354):
// stress_strain_tria3 (FEMKernels.jl:7391-7432); its shear from the
// virtual-quad macro (tria3_plate_macro_shear_resultant, :7225-7265) and, for
// shared-edge weight w > 0, the macro moment blend (_blend_tria3_macro_bending_iso!,
// stress_recovery.jl:53-86, with tria3_plate_macro_average_moment).  Both
// macros use Cm = D h, Cb = D h^3/12 and Cs = 5/6 G h with G = E / 2(1 + nu):
// the stiffness kernel's plate phases run with those scalars.  out points at
// the CTRIA3 part of the shell records.
__global__ void __launch_bounds__(T3_THREADS) t3_recover_kernel(int64_t nt, const int32_t *__restrict__ nodes,
                                                                const double *__restrict__ prop,
                                                                const double *__restrict__ coords,
                                                                const double *__restrict__ nodeR,
                                                                const double *__restrict__ u,
                                                                const double *__restrict__ mw, double *__restrict__ out) {
    __shared__ T3KShared sh[T3_ELEMS_PER_BLOCK];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane >> 4, tl = lane & 15;
    const unsigned tm = 0xFFFFu << (16 * team);
    const int64_t e = (int64_t)blockIdx.x * T3_ELEMS_PER_BLOCK + warp * T3_TEAMS_PER_WARP + team;
    if (e >= nt) return;  // the whole team leaves; syncs below are team-local
    T3KShared &S = sh[warp * T3_TEAMS_PER_WARP + team];

    // every lane: frame, local coordinates and local displacements
    const double *pr = prop + 7 * e;
    const double h = __ldg(pr), E = __ldg(pr + 1), nu = __ldg(pr + 2), br = __ldg(pr + 4);
    int32_t nd[3];
    double p[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        nd[k] = __ldg(nodes + 3 * e + k);
#pragma unroll
        for (int i = 0; i < 3; ++i) p[k][i] = __ldg(coords + 3 * (int64_t)nd[k] + i);
    }
    double V[9], x[3], y[3];
    {
        double v1[3], v2[3], v3[3], cen[3];
        t3_frame(p[0], p[1], p[2], v1, v2, v3);
        for (int i = 0; i < 3; ++i) { cen[i] = (p[0][i] + p[1][i] + p[2][i]) / 3.0; V[i] = v1[i]; V[3 + i] = v2[i]; V[6 + i] = v3[i]; }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double d[3];
            sub3(p[k], cen, d);
            x[k] = dot3(d, v1);
            y[k] = dot3(d, v2);
        }
    }
    double ul[3][6];
#pragma unroll
    for (int k = 0; k < 3; ++k) shell_node_local(V, nodeR, nd[k], u, ul[k]);
    const double A = 0.5 * fabs(x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]));
    const double c = E / (1 - nu * nu), G = E / (2.0 * (1.0 + nu));
    const double cb_r = c * (h * h * h / 12.0), cs_r = 5.0 / 6.0 * G * h;
    const bool plate = br > 1e-12 && A >= 1e-12;
    const bool macneal = plate && !(h < 1e-30 || fabs(cs_r) < 1e-30);

    // lanes 0-2: one virtual quad each -- plate dofs of its macro nodes
    // (internal ones -X u_plate), Gauss-averaged curvature, MITC4 centre
    // shear and the quad's area; S.Pb is free after the condensation
    double *qa = &S.Pb[0][0][0];
    if (plate) {
        t3_plate_points(S, tl, tm, x, y, cs_r, cb_r, macneal);
        t3_plate_blocks(S, tl, tm, cb_r, nu, (1 - nu) / 2, macneal);
        t3_condense(S, tl, tm);
        if (tl < 3) {
            const int q = tl;
            const double up[9] = {ul[0][2], ul[0][3], ul[0][4], ul[1][2], ul[1][3], ul[1][4], ul[2][2], ul[2][3], ul[2][4]};
            double lq[4][2], w[4], tx[4], ty[4];
            t3_quad_coords(q, x, y, lq);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int nid = t3_quad_node(q, k);
                if (nid < 3) {
                    w[k] = up[3 * nid]; tx[k] = up[3 * nid + 1]; ty[k] = up[3 * nid + 2];
                } else {
                    double v[3];
#pragma unroll
                    for (int dd = 0; dd < 3; ++dd) {
                        double sacc = 0.0;
#pragma unroll
                        for (int cc = 0; cc < 9; ++cc) sacc += -S.u.c.X[3 * (nid - 3) + dd][cc] * up[cc];
                        v[dd] = sacc;
                    }
                    w[k] = v[0]; tx[k] = v[1]; ty[k] = v[2];
                }
            }
            double ka[3] = {0, 0, 0}, wsum = 0.0;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                double r, s, dx[4], dy[4], iJ[4];
                q4_shape_gp(g, r, s);
                const double det = q4_point_derivs(lq, r, s, false, dx, dy, iJ);
                const double wd = fabs(det) < 1e-12 ? 1e-12 : fabs(det);
                double k0 = 0, k1 = 0, k2 = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) { k0 += dx[k] * ty[k]; k1 += -dy[k] * tx[k]; k2 += dy[k] * ty[k] - dx[k] * tx[k]; }
                ka[0] += k0 * wd; ka[1] += k1 * wd; ka[2] += k2 * wd;
                wsum += wd;
            }
            double t[3], Mq[3], Qq[2];
#pragma unroll
            for (int k = 0; k < 3; ++k) ka[k] /= wsum;
            ps_mul(c, nu, ka, t);
#pragma unroll
            for (int k = 0; k < 3; ++k) Mq[k] = -br * t[k] * (h * h * h / 12.0);
            mitc4_center_shear(lq, w, tx, ty, G, h, Qq);
            // _tria3_virtual_quad_area (FEMKernels.jl:7151-7155)
            const double a1 = (lq[1][0] - lq[0][0]) * (lq[3][1] - lq[0][1]) - (lq[3][0] - lq[0][0]) * (lq[1][1] - lq[0][1]);
            const double a2 = (lq[2][0] - lq[1][0]) * (lq[3][1] - lq[1][1]) - (lq[3][0] - lq[1][0]) * (lq[2][1] - lq[1][1]);
            const double area = (fabs(a1) + fabs(a2)) / 2;
            qa[6 * q + 0] = area * Mq[0]; qa[6 * q + 1] = area * Mq[1]; qa[6 * q + 2] = area * Mq[2];
            qa[6 * q + 3] = area * Qq[0]; qa[6 * q + 4] = area * Qq[1]; qa[6 * q + 5] = area;
        }
        __syncwarp(tm);
    }
    if (tl != 0) return;
    double *o = out + REC_SHELL * e;
    for (int i = 0; i < REC_SHELL; ++i) o[i] = 0.0;
    if (A < 1e-12) {
        o[21] = 1.0;  // degenerate triangle: the reference reports zeros
        return;
    }
    const double i2A = 1.0 / (2 * A);
    const double b[3] = {(y[1] - y[2]) * i2A, (y[2] - y[0]) * i2A, (y[0] - y[1]) * i2A};
    const double cv[3] = {(x[2] - x[1]) * i2A, (x[0] - x[2]) * i2A, (x[1] - x[0]) * i2A};
    double eps[3] = {0, 0, 0}, kap[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        eps[0] += b[i] * ul[i][0]; eps[1] += cv[i] * ul[i][1]; eps[2] += cv[i] * ul[i][0] + b[i] * ul[i][1];
        kap[0] += b[i] * ul[i][4]; kap[1] += -cv[i] * ul[i][3]; kap[2] += cv[i] * ul[i][4] - b[i] * ul[i][3];
    }
    double N[3], M[3], Q[2] = {0.0, 0.0}, t[3];
    ps_mul(c, nu, eps, t);
#pragma unroll
    for (int k = 0; k < 3; ++k) N[k] = t[k] * h;
    ps_mul(c, nu, kap, t);
#pragma unroll
    for (int k = 0; k < 3; ++k) M[k] = -br * t[k] * (h * h * h / 12.0);
    double ez1[3], ez2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { ez1[k] = eps[k] + (-h / 2.0) * kap[k]; ez2[k] = eps[k] + (h / 2.0) * kap[k]; }
    if (plate) {
        double Ms[3] = {0, 0, 0}, Qs[2] = {0, 0}, As = 0.0;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            Ms[0] += qa[6 * q]; Ms[1] += qa[6 * q + 1]; Ms[2] += qa[6 * q + 2];
            Qs[0] += qa[6 * q + 3]; Qs[1] += qa[6 * q + 4]; As += qa[6 * q + 5];
        }
        if (As > 1e-12) { Q[0] = Qs[0] / As; Q[1] = Qs[1] / As; }
        const double wgt = __ldg(mw + e);
        if (wgt > 0.0) {
            double Mm[3] = {0, 0, 0};
            if (As > 1e-12) { Mm[0] = Ms[0] / As; Mm[1] = Ms[1] / As; Mm[2] = Ms[2] / As; }
            if (isfinite(Mm[0]) && isfinite(Mm[1]) && isfinite(Mm[2])) {
                double Mb[3], kb[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) Mb[k] = (1.0 - wgt) * M[k] + wgt * Mm[k];
                // D \ M_blend with D^-1 = [1 -nu 0; -nu 1 0; 0 0 2(1 + nu)] / E
                const double di0 = (Mb[0] - nu * Mb[1]) / E, di1 = (Mb[1] - nu * Mb[0]) / E, di2 = 2.0 * (1.0 + nu) * Mb[2] / E;
                const double f = -(12.0 / (br * h * h * h));
                kb[0] = f * di0; kb[1] = f * di1; kb[2] = f * di2;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double em = (ez1[k] + ez2[k]) / 2.0;
                    M[k] = Mb[k];
                    ez1[k] = em + (-h / 2.0) * kb[k];
                    ez2[k] = em + (h / 2.0) * kb[k];
                }
            }
        }
    }
    put_shell_rec(o, N, M, Q, ez1, ez2, c, nu);
}

// CBAR/CBEAM loop body of recover_bar_stresses! (stress_recovery.jl:446-503):
// local displacements with the offset terms, forces_frame3d
// (FEMKernels.jl:215-229) and the section-point stresses.
template <int I>
__device__ __forceinline__ double frame_row(const FrameK &c, const double ub[12]) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 12; ++j)
        if (frame_nz(I, j)) s += frame_k(c, I, j) * ub[j];
    return s;
}

__global__ void __launch_bounds__(128) bar_recover_kernel(int64_t nb, const int32_t *__restrict__ nodes,
                                                          const double *__restrict__ prop,
                                                          const double *__restrict__ coords,
                                                          const double *__restrict__ nodeR, const double *__restrict__ u,
                                                          const double *__restrict__ pts, double *__restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nb) return;
    double *o = out + REC_BAR * e;
    BarFrame F;
    int32_t nd[2];
    if (!bar_frame(e, nodes, prop, coords, nodeR, F, nd)) {
        for (int i = 0; i < REC_BAR; ++i) o[i] = 0.0;  // zero-length bar: skipped by the reference
        return;
    }
    double ub[12];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        double ug[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) ug[i] = __ldg(u + 6 * (int64_t)nd[k] + i);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            double st = 0.0, sr = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                st += F.TR[k][3 * r + q] * ug[q] + F.Toff[k][3 * r + q] * ug[3 + q];
                sr += F.TR[k][3 * r + q] * ug[3 + q];
            }
            ub[6 * k + r] = st;
            ub[6 * k + 3 + r] = sr;
        }
    }
    const double *pr = prop + 18 * e;
    const FrameK c = frame3d_k(pr, F.L);
    const double f1 = frame_row<1>(c, ub), f2 = frame_row<2>(c, ub), f3 = frame_row<3>(c, ub);
    const double f4 = frame_row<4>(c, ub), f5 = frame_row<5>(c, ub), f6 = frame_row<6>(c, ub);
    const double f10 = frame_row<10>(c, ub), f11 = frame_row<11>(c, ub);
    const double A = __ldg(pr);
    double r[REC_BAR];
    r[0] = f6; r[1] = -f1; r[2] = -f2; r[3] = -f3; r[4] = -f5; r[5] = f4; r[6] = f11; r[7] = -f10;
    r[8] = fabs(A) > 1e-30 ? f6 / A : 0.0;
    double Iz = __ldg(pr + 1), Iy = __ldg(pr + 2);
    if (Iy == 0.0) Iy = Iz;
    if (Iz == 0.0) Iz = Iy;
    const double I12 = __ldg(pr + 3), den = Iz * Iy - I12 * I12;
#pragma unroll
    for (int end = 0; end < 2; ++end) {
        const double m1 = end == 0 ? r[4] : r[6], m2 = end == 0 ? r[5] : r[7];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double sv = 0.0;
            if (pts) {
                const double *pp = pts + 9 * e;
                const double yj = __ldg(pp + 2 * j), zj = __ldg(pp + 2 * j + 1);
                sv = fabs(den) > 1e-30 ? ((m1 * Iy - m2 * I12) * yj + (m2 * Iz - m1 * I12) * zj) / den
                                       : m1 * yj / fmax(Iz, 1e-30) + m2 * zj / fmax(Iy, 1e-30);
                sv *= __ldg(pp + 8);
            }
            r[9 + 4 * end + j] = sv;
        }
    }
    r[17] = 1.0;
#pragma unroll
    for (int i = 0; i < REC_BAR; ++i) o[i] = r[i];
}

// _tria3_shell_macro_blend_weights (stress_recovery.jl:20-51): every shell
// edge as a sorted-node key; a CTRIA3 edge is shared when its key occurs
// more than once.
__global__ void shell_edge_keys_kernel(int64_t nq, int64_t nt, const int32_t *__restrict__ q4n,
                                       const int32_t *__restrict__ t3n, unsigned long long *__restrict__ keys) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * nq + 3 * nt) return;
    int32_t a, b;
    if (t < 4 * nq) {
        const int64_t e = t >> 2;
        const int k = (int)(t & 3);
        a = q4n[4 * e + k]; b = q4n[4 * e + ((k + 1) & 3)];
    } else {
        const int64_t s = t - 4 * nq, e = s / 3;
        const int k = (int)(s - 3 * e);
        a = t3n[3 * e + k]; b = t3n[3 * e + (k == 2 ? 0 : k + 1)];
    }
    const uint32_t lo = (uint32_t)min(a, b), hi = (uint32_t)max(a, b);
    keys[t] = ((unsigned long long)lo << 32) | hi;
}

__device__ __forceinline__ int64_t key_count(const unsigned long long *__restrict__ k, int64_t n, unsigned long long key) {
    int64_t lo = 0, hi = n;  // first index >= key
    while (lo < hi) { const int64_t m = (lo + hi) >> 1; if (k[m] < key) lo = m + 1; else hi = m; }
    int64_t lo2 = lo, hi2 = n;  // first index > key
    while (lo2 < hi2) { const int64_t m = (lo2 + hi2) >> 1; if (k[m] <= key) lo2 = m + 1; else hi2 = m; }
    return lo2 - lo;
}

__global__ void t3_macro_weight_kernel(int64_t nt, const int32_t *__restrict__ t3n,
                                       const unsigned long long *__restrict__ sorted, int64_t n_keys,
                                       double *__restrict__ w) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nt) return;
    int shared = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int32_t a = t3n[3 * e + k], b = t3n[3 * e + (k == 2 ? 0 : k + 1)];
        const uint32_t lo = (uint32_t)min(a, b), hi = (uint32_t)max(a, b);
        shared += key_count(sorted, n_keys, ((unsigned long long)lo << 32) | hi) > 1;
    }
    w[e] = fmin(1.0, fmax(0.0, (shared - 1) / 2.0));
}

}  // namespace jfg
