// jfem_oracle.cpp -- CPU restatement of the OpenJFEM element hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
// baseline; nothing in the product library links or calls it.  It restates,
// in plain C++ with OpenMP over elements, the default branch of
//   assemble_stiffness            src/solver/assembly.jl:1953-4375
//   assemble_geometric_stiffness  src/solver/assembly.jl:4382-6634
// and the element kernels they call in src/FEMKernels.jl, restricted to the
// predicates the library accepts (flat isotropic PSHELL/MAT1 CQUAD4/CTRIA3,
// CBAR/CBEAM without pin flags, RBE2, PARAM SNORM <= 0, no JFEM_* overrides).
//
// PARITY UNPINNED: the reference is Julia 1.12 and cannot run where this
// library is built and tested (no julia, no network), and it ships no golden vectors or
// known-answer tests for this path.  The restatement follows the cited lines;
// agreement with it is checked by tests, and physics known-answers (symmetry,
// rigid-body null space, plate buckling coefficient) add sanity checks that
// are not reference-pinned.
//
// Third-party arithmetic restated here (not vendored in the reference):
//   StaticArrays 1.9.17 inv(SMatrix{4,4})     -> Gauss-Jordan with pivoting
//   LinearAlgebra (OpenBLAS 0.3.29) small '\' -> LU with partial pivoting
//   SparseArrays 1.12.0 sparse(I,J,V,m,n)     -> CSC, duplicates summed,
//                                                 explicit zeros kept
// They differ from the reference only by rounding.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/jfem_gpu.h"

namespace {

typedef double V3[3];

// Forward-mode dual number v + d eps (eps^2 = 0): the oracle's restatement of
// ForwardDiff's Dual with one partial, which the reference uses to
// differentiate the shell elements in their thickness (dKdx.jl:219-228).
// Comparisons and branches look at the value only, as ForwardDiff's do.
struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double x) : v(x), d(0.0) {}  // NOLINT: constants promote implicitly
    Dual(double x, double dx) : v(x), d(dx) {}
    Dual &operator+=(const Dual &o) { v += o.v; d += o.d; return *this; }
    Dual &operator-=(const Dual &o) { v -= o.v; d -= o.d; return *this; }
    Dual &operator*=(const Dual &o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
    Dual &operator/=(const Dual &o) { *this = Dual(v / o.v, (d * o.v - v * o.d) / (o.v * o.v)); return *this; }
};
inline Dual operator+(Dual a, const Dual &b) { return a += b; }
inline Dual operator-(Dual a, const Dual &b) { return a -= b; }
inline Dual operator*(Dual a, const Dual &b) { return a *= b; }
inline Dual operator/(Dual a, const Dual &b) { return a /= b; }
inline Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
inline bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
inline bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
inline bool operator==(const Dual &a, const Dual &b) { return a.v == b.v; }
inline Dual fabs(const Dual &a) { return a.v < 0.0 ? -a : a; }
inline Dual sqrt(const Dual &a) { const double r = std::sqrt(a.v); return Dual(r, a.d / (2.0 * r)); }
inline double value(double x) { return x; }
inline double value(const Dual &x) { return x.v; }
// max(|x|, floor) with the derivative of the branch taken
template <typename T> inline T abs_floor(const T &x, double floor) {
    using std::fabs;
    const T a = fabs(x);
    return value(a) < floor ? T(floor) : a;
}


inline void sub3(const double *a, const double *b, double *o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }
inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross3(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
inline double norm3(const double *a) { return std::sqrt(dot3(a, a)); }
inline void normalize3(const double *a, double *o) { double n = norm3(a); o[0] = a[0] / n; o[1] = a[1] / n; o[2] = a[2] / n; }

// Dense LU with partial pivoting: solve A X = B in place (A n x n, B n x m),
// row-major.  Returns false on an exactly singular pivot.
template <typename T>
bool lu_solve(int n, int m, T *A, T *B) {
    using std::fabs;
    for (int k = 0; k < n; ++k) {
        int p = k;
        T best = fabs(A[k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            T v = fabs(A[i * n + k]);
            if (v > best) { best = v; p = i; }
        }
        if (value(best) == 0.0) return false;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
            for (int j = 0; j < m; ++j) std::swap(B[k * m + j], B[p * m + j]);
        }
        for (int i = k + 1; i < n; ++i) {
            T f = A[i * n + k] / A[k * n + k];
            A[i * n + k] = f;
            for (int j = k + 1; j < n; ++j) A[i * n + j] -= f * A[k * n + j];
            for (int j = 0; j < m; ++j) B[i * m + j] -= f * B[k * m + j];
        }
    }
    for (int k = n - 1; k >= 0; --k) {
        for (int j = 0; j < m; ++j) {
            T s = B[k * m + j];
            for (int i = k + 1; i < n; ++i) s -= A[k * n + i] * B[i * m + j];
            B[k * m + j] = s / A[k * n + k];
        }
    }
    return true;
}

// inv(SMatrix{4,4}) restated as Gauss-Jordan (identity right-hand side).
template <typename T>
void inv4(const T A[4][4], T Ai[4][4]) {
    T a[16], b[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) { a[i * 4 + j] = A[i][j]; b[i * 4 + j] = (i == j) ? 1.0 : 0.0; }
    lu_solve(4, 4, a, b);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Ai[i][j] = b[i * 4 + j];
}

// shape_derivs_quad (FEMKernels.jl:237-241)
inline void shape_derivs_quad(double xi, double eta, double dNr[4], double dNs[4]) {
    dNr[0] = -0.25 * (1 - eta); dNr[1] = 0.25 * (1 - eta); dNr[2] = 0.25 * (1 + eta); dNr[3] = -0.25 * (1 + eta);
    dNs[0] = -0.25 * (1 - xi); dNs[1] = -0.25 * (1 + xi); dNs[2] = 0.25 * (1 + xi); dNs[3] = 0.25 * (1 - xi);
}

struct Jac {
    double J11, J12, J21, J22, det, iJ11, iJ12, iJ21, iJ22;
};
inline Jac jacobian(const double lc[4][2], const double dNr[4], const double dNs[4]) {
    Jac j;
    j.J11 = dNr[0] * lc[0][0] + dNr[1] * lc[1][0] + dNr[2] * lc[2][0] + dNr[3] * lc[3][0];
    j.J12 = dNr[0] * lc[0][1] + dNr[1] * lc[1][1] + dNr[2] * lc[2][1] + dNr[3] * lc[3][1];
    j.J21 = dNs[0] * lc[0][0] + dNs[1] * lc[1][0] + dNs[2] * lc[2][0] + dNs[3] * lc[3][0];
    j.J22 = dNs[0] * lc[0][1] + dNs[1] * lc[1][1] + dNs[2] * lc[2][1] + dNs[3] * lc[3][1];
    j.det = j.J11 * j.J22 - j.J12 * j.J21;
    double inv = 1.0 / j.det;
    j.iJ11 = j.J22 * inv; j.iJ12 = -j.J12 * inv; j.iJ21 = -j.J21 * inv; j.iJ22 = j.J11 * inv;
    return j;
}

// C += alpha * A' * B  with A (k x m), B (k x n), C (m x n), all row-major.
template <typename TC, typename TA, typename TB, typename TS>
void mul_At_add(TC *C, const TA *A, const TB *B, int k, int m, int n, TS alpha) {
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < k; ++l) {
            TC v = alpha * B[l * n + j];
            for (int i = 0; i < m; ++i) C[i * n + j] += A[l * m + i] * v;
        }
}
// C = A * B  (A m x k, B k x n)
template <typename TC, typename TA, typename TB>
void mul(TC *C, const TA *A, const TB *B, int m, int k, int n) {
    for (int i = 0; i < m * n; ++i) C[i] = 0.0;
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < k; ++l) {
            TC v = B[l * n + j];
            for (int i = 0; i < m; ++i) C[i * n + j] += A[i * k + l] * v;
        }
}

// add_quad4_macneal_shear_rbf! default branch (FEMKernels.jl:4715-4978):
// epsilon 0.04, "diag" flexibility, paper length mode, zb_scale 0.65,
// zb_u = zb_d, no per-GP delta, rigid_shear = false.
template <typename T>
void macneal_shear(T Ke[24][24], const double lc[4][2], const T Cb[3][3], const T Cs[2][2], T h) {
    using std::fabs;
    const double csmax = std::max(std::max(std::fabs(value(Cs[0][0])), std::fabs(value(Cs[0][1]))),
                                  std::max(std::fabs(value(Cs[1][0])), std::fabs(value(Cs[1][1]))));
    if (value(h) < 1e-30 || csmax < 1e-30) return;
    const double pt = 1.0 / std::sqrt(3.0);
    const double sp[4][3] = {{0.0, -pt, 1}, {0.0, pt, 1}, {-pt, 0.0, 2}, {pt, 0.0, 2}};
    double D[4][12] = {};
    double Jp[4];
    for (int s = 0; s < 4; ++s) {
        double xi = sp[s][0], eta = sp[s][1];
        int comp = (int)sp[s][2];
        double dNr[4], dNs[4];
        shape_derivs_quad(xi, eta, dNr, dNs);
        double J11 = dNr[0] * lc[0][0] + dNr[1] * lc[1][0] + dNr[2] * lc[2][0] + dNr[3] * lc[3][0];
        double J12 = dNr[0] * lc[0][1] + dNr[1] * lc[1][1] + dNr[2] * lc[2][1] + dNr[3] * lc[3][1];
        double J21 = dNs[0] * lc[0][0] + dNs[1] * lc[1][0] + dNs[2] * lc[2][0] + dNs[3] * lc[3][0];
        double J22 = dNs[0] * lc[0][1] + dNs[1] * lc[1][1] + dNs[2] * lc[2][1] + dNs[3] * lc[3][1];
        double det = J11 * J22 - J12 * J21;
        if (std::fabs(det) < 1e-14) det = det < 0.0 ? -1e-14 : 1e-14;
        Jp[s] = std::fabs(det);
        double inv = 1.0 / det;
        double iJ11 = J22 * inv, iJ12 = -J12 * inv, iJ21 = -J21 * inv, iJ22 = J11 * inv;
        double N[4] = {0.25 * (1 - xi) * (1 - eta), 0.25 * (1 + xi) * (1 - eta), 0.25 * (1 + xi) * (1 + eta), 0.25 * (1 - xi) * (1 + eta)};
        for (int k = 0; k < 4; ++k) {
            double dx = iJ11 * dNr[k] + iJ12 * dNs[k];
            double dy = iJ21 * dNr[k] + iJ22 * dNs[k];
            int col = 3 * k;
            if (comp == 1) { D[s][col + 0] = dx; D[s][col + 2] = N[k]; }
            else { D[s][col + 0] = dy; D[s][col + 1] = -N[k]; }
        }
    }
    double Dx = 0.5 * (lc[1][0] + lc[2][0] - lc[0][0] - lc[3][0]);
    double Dy = 0.5 * (lc[2][1] + lc[3][1] - lc[0][1] - lc[1][1]);
    double Dx2 = Dx * Dx, Dy2 = Dy * Dy;
    const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25}, dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
    double J11c = dNr_c[0] * lc[0][0] + dNr_c[1] * lc[1][0] + dNr_c[2] * lc[2][0] + dNr_c[3] * lc[3][0];
    double J12c = dNr_c[0] * lc[0][1] + dNr_c[1] * lc[1][1] + dNr_c[2] * lc[2][1] + dNr_c[3] * lc[3][1];
    double J21c = dNs_c[0] * lc[0][0] + dNs_c[1] * lc[1][0] + dNs_c[2] * lc[2][0] + dNs_c[3] * lc[3][0];
    double J22c = dNs_c[0] * lc[0][1] + dNs_c[1] * lc[1][1] + dNs_c[2] * lc[2][1] + dNs_c[3] * lc[3][1];
    double A_elem = 4.0 * std::fabs(J11c * J22c - J12c * J21c);
    double eps = std::min(std::max(0.04, 1e-12), 1.0);
    double a_param = eps / (eps + (1.0 - eps) * Dx2 / std::max(Dy2, 1e-30));
    double b_param = eps / (eps + (1.0 - eps) * Dy2 / std::max(Dx2, 1e-30));
    T flex_x = 1.0 / abs_floor(Cb[0][0], 1e-30);
    T flex_y = 1.0 / abs_floor(Cb[1][1], 1e-30);
    double inv12A = 1.0 / (12.0 * A_elem);
    const double zb = 0.65;
    T zbx_u = zb * inv12A * Dx2 * flex_x;
    T zbx_d = zb * inv12A * a_param * Dx2 * flex_x;
    T zby_u = zb * inv12A * Dy2 * flex_y;
    T zby_d = zb * inv12A * b_param * Dy2 * flex_y;
    T Zb[4][4] = {};
    Zb[0][0] = zbx_u + zbx_d; Zb[0][1] = zbx_u - zbx_d; Zb[1][0] = Zb[0][1]; Zb[1][1] = Zb[0][0];
    Zb[2][2] = zby_u + zby_d; Zb[2][3] = zby_u - zby_d; Zb[3][2] = Zb[2][3]; Zb[3][3] = Zb[2][2];
    // physical shear compliance (eq 23-25)
    const int comps[4] = {1, 1, 2, 2};
    T VGV[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double Jfac = std::sqrt(2.0 * Jp[i]) * std::sqrt(2.0 * Jp[j]);
            if (comps[i] == comps[j]) VGV[i][j] = (i == j) ? Jfac * (comps[i] == 1 ? Cs[0][0] : Cs[1][1]) : T(0.0);
            else VGV[i][j] = 0.5 * Jfac * Cs[0][1];
        }
    for (int i = 0; i < 4; ++i)
        if (value(VGV[i][i]) < 1e-30) VGV[i][i] = 1e-30;
    T VS[4][4], Zs[4][4], Zi[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) VS[i][j] = 0.5 * (VGV[i][j] + VGV[j][i]);
    inv4(VS, Zi);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Zs[i][j] = 0.5 * (Zi[i][j] + Zi[j][i]);
    T Zt[4][4], Z[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Zt[i][j] = Zs[i][j] + Zb[i][j];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Z[i * 4 + j] = 0.5 * (Zt[i][j] + Zt[j][i]);
    T X[4 * 12];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 12; ++j) X[i * 12 + j] = D[i][j];
    lu_solve(4, 12, Z, X);
    T Kp[12][12];
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) {
            T s = 0.0;
            for (int l = 0; l < 4; ++l) s += D[l][i] * X[l * 12 + j];
            Kp[i][j] = s;
        }
    const int pd[12] = {2, 3, 4, 8, 9, 10, 14, 15, 16, 20, 21, 22};
    for (int j = 0; j < 12; ++j)
        for (int i = 0; i < 12; ++i) Ke[pd[i]][pd[j]] += 0.5 * (Kp[i][j] + Kp[j][i]);
}

// stiffness_quad4_matrices, default branch (FEMKernels.jl:3185-4034) for a
// planar element: JFEM_Q4_KERNEL=macneal with the twist correction
// (:3466-3492), MITC4 shear skipped (:3762), Hughes-Brezzi drill
// (:3556-3559), Wilson incompatible modes and 4x4 condensations
// (:3790-3801, :3964-4011).  No Bmb, no curvature terms.
template <typename T>
void q4_stiffness(const double lc[4][2], const T Cm[3][3], const T Cb[3][3], const T Cs[2][2],
                  T h, T E_ref, double k6rot, double drill_scale, bool bending_incomp,
                  bool membrane_incomp, T Ke[24][24]) {
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) Ke[i][j] = 0.0;
    T K_ab[24][4] = {}, K_bb[4][4] = {}, K_abb[24][4] = {}, K_bbb[4][4] = {};
    const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25}, dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
    Jac jc = jacobian(lc, dNr_c, dNs_c);
    double dNdx_c[4], dNdy_c[4];
    for (int k = 0; k < 4; ++k) {
        dNdx_c[k] = jc.iJ11 * dNr_c[k] + jc.iJ12 * dNs_c[k];
        dNdy_c[k] = jc.iJ21 * dNr_c[k] + jc.iJ22 * dNs_c[k];
    }
    const double pt = 1.0 / std::sqrt(3.0);
    const double gp[4][2] = {{-pt, -pt}, {pt, -pt}, {pt, pt}, {-pt, pt}};
    T G_drill = Cm[2][2] / h;
    if (value(G_drill) < 1e-6) G_drill = E_ref / (2 * 3.0);
    T alpha_drill = drill_scale * (k6rot / 1e5) * G_drill * h;

    for (int g = 0; g < 4; ++g) {
        double r = gp[g][0], s = gp[g][1];
        double dNr[4], dNs[4];
        shape_derivs_quad(r, s, dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        double absdet = std::fabs(j.det);
        if (absdet < 1e-12) absdet = 1e-12;
        double Bm[3][24] = {}, Bb[3][24] = {}, Bd[1][24] = {};
        for (int k = 0; k < 4; ++k) {
            double dx = j.iJ11 * dNr[k] + j.iJ12 * dNs[k];
            double dy = j.iJ21 * dNr[k] + j.iJ22 * dNs[k];
            int idx = 6 * k;
            double Nk = 0.25 * (1 + ((k == 1 || k == 2) ? r : -r)) * (1 + (k >= 2 ? s : -s));
            Bm[0][idx + 0] = dx; Bm[1][idx + 1] = dy;
            Bm[2][idx + 0] = dy; Bm[2][idx + 1] = dx;
            Bb[0][idx + 4] = dx; Bb[1][idx + 3] = -dy;
            // MacNeal twist compatibility: 2 chi_xy(gp) - chi_xy(0)
            Bb[2][idx + 4] = 2.0 * dy - dNdy_c[k];
            Bb[2][idx + 3] = 2.0 * (-dx) - (-dNdx_c[k]);
            Bd[0][idx + 0] = 0.5 * dy; Bd[0][idx + 1] = -0.5 * dx; Bd[0][idx + 5] = Nk;
        }
        double dphi1_dx = j.iJ11 * (-2.0 * r), dphi1_dy = j.iJ21 * (-2.0 * r);
        double dphi2_dx = j.iJ12 * (-2.0 * s), dphi2_dy = j.iJ22 * (-2.0 * s);
        double Bi[3][4] = {}, Bib[3][4] = {};
        Bi[0][0] = dphi1_dx; Bi[2][0] = dphi1_dy; Bi[1][1] = dphi1_dy; Bi[2][1] = dphi1_dx;
        Bi[0][2] = dphi2_dx; Bi[2][2] = dphi2_dy; Bi[1][3] = dphi2_dy; Bi[2][3] = dphi2_dx;
        Bib[1][0] = -dphi1_dy; Bib[1][1] = -dphi2_dy;
        Bib[0][2] = dphi1_dx; Bib[0][3] = dphi2_dx;
        Bib[2][0] = -dphi1_dx; Bib[2][1] = -dphi2_dx;
        Bib[2][2] = dphi1_dy; Bib[2][3] = dphi2_dy;
        T t3x24[3 * 24], t3x4[3 * 4];
        mul(t3x24, &Cm[0][0], &Bm[0][0], 3, 3, 24);
        mul_At_add(&Ke[0][0], &Bm[0][0], t3x24, 3, 24, 24, absdet);
        mul(t3x24, &Cb[0][0], &Bb[0][0], 3, 3, 24);
        mul_At_add(&Ke[0][0], &Bb[0][0], t3x24, 3, 24, 24, absdet);
        mul_At_add(&Ke[0][0], &Bd[0][0], &Bd[0][0], 1, 24, 24, absdet * alpha_drill);
        if (membrane_incomp) {
            mul(t3x4, &Cm[0][0], &Bi[0][0], 3, 3, 4);
            mul_At_add(&K_ab[0][0], &Bm[0][0], t3x4, 3, 24, 4, absdet);
            mul_At_add(&K_bb[0][0], &Bi[0][0], t3x4, 3, 4, 4, absdet);
        }
        mul(t3x4, &Cb[0][0], &Bib[0][0], 3, 3, 4);
        mul_At_add(&K_abb[0][0], &Bb[0][0], t3x4, 3, 24, 4, absdet);
        mul_At_add(&K_bbb[0][0], &Bib[0][0], t3x4, 3, 4, 4, absdet);
    }
    macneal_shear(Ke, lc, Cb, Cs, h);

    double kbbmax = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int jj = 0; jj < 4; ++jj) kbbmax = std::max(kbbmax, std::fabs(value(K_bbb[i][jj])));
    auto condense = [&](T Kab[24][4], T Kbb[4][4]) {
        T Ii[4][4];
        inv4(Kbb, Ii);
        for (int jj = 0; jj < 24; ++jj)
            for (int i = 0; i < 24; ++i) {
                T sm = 0.0;
                for (int l = 0; l < 4; ++l) {
                    T t = 0.0;
                    for (int q = 0; q < 4; ++q) t += Ii[l][q] * Kab[jj][q];
                    sm += Kab[i][l] * t;
                }
                Ke[i][jj] -= sm;
            }
    };
    if (bending_incomp && kbbmax > 0.0) {
        condense(K_abb, K_bbb);
        if (membrane_incomp) condense(K_ab, K_bb);
    } else if (membrane_incomp) {
        condense(K_ab, K_bb);
    }
}

// stiffness_tria3_matrices_generic (FEMKernels.jl:7315-7385) with
// tria3_plate_macro_data (:7157-7209): CST membrane, plate block from three
// default-kwarg virtual quads condensed to the corners, Hughes-Brezzi drill.
template <typename T>
void t3_stiffness(const double lc[3][2], const T Dm[3][3], const T Db[3][3], const T Ds[2][2],
                  T h, T G_ref, double br, double k6rot, T Ke[18][18]) {
    for (int i = 0; i < 18; ++i)
        for (int j = 0; j < 18; ++j) Ke[i][j] = 0.0;
    double x[3] = {lc[0][0], lc[1][0], lc[2][0]}, y[3] = {lc[0][1], lc[1][1], lc[2][1]};
    double A2 = x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]);
    double A = 0.5 * std::fabs(A2);
    if (A < 1e-12) return;
    double bv[3] = {(y[1] - y[2]) / (2 * A), (y[2] - y[0]) / (2 * A), (y[0] - y[1]) / (2 * A)};
    double cv[3] = {(x[2] - x[1]) / (2 * A), (x[0] - x[2]) / (2 * A), (x[1] - x[0]) / (2 * A)};
    double Bm[3][6] = {};
    for (int i = 0; i < 3; ++i) {
        Bm[0][2 * i] = bv[i]; Bm[1][2 * i + 1] = cv[i]; Bm[2][2 * i] = cv[i]; Bm[2][2 * i + 1] = bv[i];
    }
    T DB[3 * 6], Km[6 * 6] = {};
    mul(DB, &Dm[0][0], &Bm[0][0], 3, 3, 6);
    mul_At_add(Km, &Bm[0][0], DB, 3, 6, 6, A);
    const int m_idx[6] = {0, 1, 6, 7, 12, 13};
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) Ke[m_idx[i]][m_idx[j]] = Km[i * 6 + j];
    // plate macro data
    if (br > 1e-12) {
        double pts[7][2];
        for (int i = 0; i < 3; ++i) { pts[i][0] = x[i]; pts[i][1] = y[i]; }
        pts[3][0] = (x[0] + x[1]) / 2; pts[3][1] = (y[0] + y[1]) / 2;
        pts[4][0] = (x[1] + x[2]) / 2; pts[4][1] = (y[1] + y[2]) / 2;
        pts[5][0] = (x[2] + x[0]) / 2; pts[5][1] = (y[2] + y[0]) / 2;
        pts[6][0] = (x[0] + x[1] + x[2]) / 3; pts[6][1] = (y[0] + y[1] + y[2]) / 3;
        const int quads[3][4] = {{0, 3, 6, 5}, {1, 4, 6, 3}, {2, 5, 6, 4}};
        const int pd[12] = {2, 3, 4, 8, 9, 10, 14, 15, 16, 20, 21, 22};
        static thread_local T K21[21][21];
        for (int i = 0; i < 21; ++i)
            for (int j = 0; j < 21; ++j) K21[i][j] = 0.0;
        for (int q = 0; q < 3; ++q) {
            double qc[4][2];
            for (int k = 0; k < 4; ++k) { qc[k][0] = pts[quads[q][k]][0]; qc[k][1] = pts[quads[q][k]][1]; }
            T Kq[24][24];
            q4_stiffness(qc, Dm, Db, Ds, h, G_ref, k6rot, 1.0, /*bending_incomp=*/false, /*membrane_incomp=*/true, Kq);
            int ed[12];
            for (int k = 0; k < 4; ++k)
                for (int d = 0; d < 3; ++d) ed[3 * k + d] = 3 * quads[q][k] + d;
            for (int i = 0; i < 12; ++i)
                for (int j = 0; j < 12; ++j) K21[ed[i]][ed[j]] += Kq[pd[i]][pd[j]];
        }
        T Kii[12 * 12], Aint[12 * 9];
        for (int i = 0; i < 12; ++i) {
            for (int j = 0; j < 12; ++j) Kii[i * 12 + j] = K21[9 + i][9 + j];
            for (int j = 0; j < 9; ++j) Aint[i * 9 + j] = K21[9 + i][j];
        }
        lu_solve(12, 9, Kii, Aint);
        for (int i = 0; i < 12 * 9; ++i) Aint[i] = -Aint[i];
        const int b_idx[9] = {2, 3, 4, 8, 9, 10, 14, 15, 16};
        for (int i = 0; i < 9; ++i)
            for (int j = 0; j < 9; ++j) {
                T s = K21[i][j];
                for (int l = 0; l < 12; ++l) s += K21[i][9 + l] * Aint[l * 9 + j];
                Ke[b_idx[i]][b_idx[j]] += s;
            }
    }
    T alpha_drill = (k6rot / 1e5) * G_ref * h;
    double Bd[18] = {};
    for (int i = 0; i < 3; ++i) {
        Bd[6 * i + 0] = 0.5 * cv[i]; Bd[6 * i + 1] = -0.5 * bv[i]; Bd[6 * i + 5] = 1.0 / 3.0;
    }
    for (int i = 0; i < 18; ++i)
        for (int j = 0; j < 18; ++j) Ke[i][j] += alpha_drill * (Bd[i] * Bd[j]) * A;
}

// stiffness_frame3d_generic (FEMKernels.jl:140-209)
void frame3d_stiffness(double L, double A, double Iy, double Iz, double J, double E, double G, double As_y,
                       double As_z, double I12, double k[12][12]) {
    std::memset(k, 0, sizeof(double) * 144);
    if (L < 1e-9) return;
    double X = E * A / L;
    k[0][0] = X; k[0][6] = -X; k[6][0] = -X; k[6][6] = X;
    double T = G * J / L;
    k[3][3] = T; k[3][9] = -T; k[9][3] = -T; k[9][9] = T;
    double Phi_y = std::isinf(As_z) ? 0.0 : 12 * E * Iy / (G * As_z * L * L);
    double Phi_z = std::isinf(As_y) ? 0.0 : 12 * E * Iz / (G * As_y * L * L);
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
    if (std::fabs(I12) > 0.0) {
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

// quad4_membrane_force_field with incompatible modes (FEMKernels.jl:6341-6539)
void q4_membrane_force_field(const double lc[4][2], const double u[24], const double Cm[3][3], double Ngp[4][3]) {
    const double pt = 1.0 / std::sqrt(3.0);
    const double gp[4][2] = {{-pt, -pt}, {pt, -pt}, {pt, pt}, {-pt, pt}};
    double K_ab[24][4] = {}, K_bb[4][4] = {};
    double Bm_g[4][3][24], Bi_g[4][3][4];
    for (int g = 0; g < 4; ++g) {
        double r = gp[g][0], s = gp[g][1];
        double dNr[4], dNs[4];
        shape_derivs_quad(r, s, dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        double detg = std::fabs(j.det);
        if (detg < 1e-12) detg = 1e-12;
        std::memset(Bm_g[g], 0, sizeof(Bm_g[g]));
        std::memset(Bi_g[g], 0, sizeof(Bi_g[g]));
        for (int k = 0; k < 4; ++k) {
            double dx = j.iJ11 * dNr[k] + j.iJ12 * dNs[k];
            double dy = j.iJ21 * dNr[k] + j.iJ22 * dNs[k];
            Bm_g[g][0][6 * k] = dx; Bm_g[g][1][6 * k + 1] = dy; Bm_g[g][2][6 * k] = dy; Bm_g[g][2][6 * k + 1] = dx;
        }
        double d1x = j.iJ11 * (-2.0 * r), d1y = j.iJ21 * (-2.0 * r), d2x = j.iJ12 * (-2.0 * s), d2y = j.iJ22 * (-2.0 * s);
        Bi_g[g][0][0] = d1x; Bi_g[g][2][0] = d1y; Bi_g[g][1][1] = d1y; Bi_g[g][2][1] = d1x;
        Bi_g[g][0][2] = d2x; Bi_g[g][2][2] = d2y; Bi_g[g][1][3] = d2y; Bi_g[g][2][3] = d2x;
        double CBi[3 * 4];
        mul(CBi, &Cm[0][0], &Bi_g[g][0][0], 3, 3, 4);
        mul_At_add(&K_ab[0][0], &Bm_g[g][0][0], CBi, 3, 24, 4, detg);
        mul_At_add(&K_bb[0][0], &Bi_g[g][0][0], CBi, 3, 4, 4, detg);
    }
    double rhs[4], A[16];
    for (int l = 0; l < 4; ++l) {
        double s = 0.0;
        for (int i = 0; i < 24; ++i) s += K_ab[i][l] * u[i];
        rhs[l] = s;
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) A[i * 4 + j] = K_bb[i][j];
    lu_solve(4, 1, A, rhs);
    double alpha[4] = {-rhs[0], -rhs[1], -rhs[2], -rhs[3]};
    for (int g = 0; g < 4; ++g) {
        double eps[3];
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int i = 0; i < 24; ++i) s += Bm_g[g][c][i] * u[i];
            for (int l = 0; l < 4; ++l) s += Bi_g[g][c][l] * alpha[l];
            eps[c] = s;
        }
        for (int c = 0; c < 3; ++c) Ngp[g][c] = Cm[c][0] * eps[0] + Cm[c][1] * eps[1] + Cm[c][2] * eps[2];
    }
}

// quad4_membrane_incompatible_condensation_map (FEMKernels.jl:6708-6785):
// returns A = -(K_bb \ K_ab') (4 x 24).
void q4_incomp_map(const double lc[4][2], const double Cm[3][3], double Amap[4][24]) {
    const double pt = 1.0 / std::sqrt(3.0);
    const double gp[4][2] = {{-pt, -pt}, {pt, -pt}, {pt, pt}, {-pt, pt}};
    double K_ab[24][4] = {}, K_bb[4][4] = {};
    for (int g = 0; g < 4; ++g) {
        double r = gp[g][0], s = gp[g][1];
        double dNr[4], dNs[4];
        shape_derivs_quad(r, s, dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        double detg = std::fabs(j.det);
        if (detg < 1e-12) detg = 1e-12;
        double Bm[3][24] = {}, Bi[3][4] = {};
        for (int k = 0; k < 4; ++k) {
            double dx = j.iJ11 * dNr[k] + j.iJ12 * dNs[k];
            double dy = j.iJ21 * dNr[k] + j.iJ22 * dNs[k];
            Bm[0][6 * k] = dx; Bm[1][6 * k + 1] = dy; Bm[2][6 * k] = dy; Bm[2][6 * k + 1] = dx;
        }
        double d1x = j.iJ11 * (-2.0 * r), d1y = j.iJ21 * (-2.0 * r), d2x = j.iJ12 * (-2.0 * s), d2y = j.iJ22 * (-2.0 * s);
        Bi[0][0] = d1x; Bi[2][0] = d1y; Bi[1][1] = d1y; Bi[2][1] = d1x;
        Bi[0][2] = d2x; Bi[2][2] = d2y; Bi[1][3] = d2y; Bi[2][3] = d2x;
        double CBi[12];
        mul(CBi, &Cm[0][0], &Bi[0][0], 3, 3, 4);
        mul_At_add(&K_ab[0][0], &Bm[0][0], CBi, 3, 24, 4, detg);
        mul_At_add(&K_bb[0][0], &Bi[0][0], CBi, 3, 4, 4, detg);
    }
    double A[16], B[4 * 24];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) A[i * 4 + j] = K_bb[i][j];
    for (int l = 0; l < 4; ++l)
        for (int i = 0; i < 24; ++i) B[l * 24 + i] = K_ab[i][l];
    lu_solve(4, 24, A, B);
    for (int l = 0; l < 4; ++l)
        for (int i = 0; i < 24; ++i) Amap[l][i] = -B[l * 24 + i];
}

// principal_stress_2d_components (FEMKernels.jl:6891-6902)
void principal2d(double sxx, double syy, double sxy, double out[6]) {
    double mean = 0.5 * (sxx + syy), hd = 0.5 * (sxx - syy);
    double rad = std::sqrt(hd * hd + sxy * sxy);
    if (rad <= 1e-30) { out[0] = mean; out[1] = 1.0; out[2] = 0.0; out[3] = mean; out[4] = 0.0; out[5] = 1.0; return; }
    double th = 0.5 * std::atan2(2.0 * sxy, sxx - syy);
    double c = std::cos(th), s = std::sin(th);
    out[0] = mean + rad; out[1] = c; out[2] = s; out[3] = mean - rad; out[4] = -s; out[5] = c;
}

// geometric_stiffness_quad4 (matrix-sigma method, FEMKernels.jl:7554-7985)
// with trans_mode = :principal_transverse, membrane_incomp = true,
// rot_grad_scale = 0 (flat), shear factors 1.
void q4_geometric_stiffness(const double lc[4][2], const double sig[4][3], double h, const double Cm[3][3],
                            double Kg[24][24]) {
    std::memset(Kg, 0, sizeof(double) * 576);
    if (h < 1e-30) return;
    double Amap[4][24];
    q4_incomp_map(lc, Cm, Amap);
    const double pt = 1.0 / std::sqrt(3.0);
    const double gp[4][2] = {{-pt, -pt}, {pt, -pt}, {pt, pt}, {-pt, pt}};
    for (int g = 0; g < 4; ++g) {
        double sxx = sig[g][0], syy = sig[g][1], sxy = sig[g][2];
        double r = gp[g][0], s = gp[g][1];
        double dNr[4], dNs[4];
        shape_derivs_quad(r, s, dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        double absdet = std::fabs(j.det);
        if (absdet < 1e-12) absdet = 1e-12;
        double uxx[24] = {}, uxy[24] = {}, uyx[24] = {}, uyy[24] = {}, uzx[24] = {}, uzy[24] = {};
        for (int i = 0; i < 4; ++i) {
            double dx = j.iJ11 * dNr[i] + j.iJ12 * dNs[i];
            double dy = j.iJ21 * dNr[i] + j.iJ22 * dNs[i];
            int r0 = 6 * i;
            uxx[r0] = dx; uxy[r0] = dy; uyx[r0 + 1] = dx; uyy[r0 + 1] = dy; uzx[r0 + 2] = dx; uzy[r0 + 2] = dy;
        }
        double d1x = j.iJ11 * (-2.0 * r), d1y = j.iJ21 * (-2.0 * r), d2x = j.iJ12 * (-2.0 * s), d2y = j.iJ22 * (-2.0 * s);
        for (int a = 0; a < 24; ++a) {
            double a1 = Amap[0][a], a2 = Amap[1][a], a3 = Amap[2][a], a4 = Amap[3][a];
            uxx[a] += d1x * a1 + d2x * a3;
            uxy[a] += d1y * a1 + d2y * a3;
            uyx[a] += d1x * a2 + d2x * a4;
            uyy[a] += d1y * a2 + d2y * a4;
        }
        double scale = h * absdet;
        double pr[6];
        principal2d(sxx, syy, sxy, pr);
        for (int dir = 0; dir < 2; ++dir) {
            double lam = pr[3 * dir], c = pr[3 * dir + 1], sn = pr[3 * dir + 2];
            if (std::fabs(lam) <= 1e-30) continue;
            double p11 = sn * sn, p22 = c * c, p12 = -c * sn;
            double f = scale * lam;
            for (int jj = 0; jj < 24; ++jj) {
                double gxj = c * uxx[jj] + sn * uxy[jj], gyj = c * uyx[jj] + sn * uyy[jj], gzj = c * uzx[jj] + sn * uzy[jj];
                for (int ii = 0; ii < 24; ++ii) {
                    double gxi = c * uxx[ii] + sn * uxy[ii], gyi = c * uyx[ii] + sn * uyy[ii], gzi = c * uzx[ii] + sn * uzy[ii];
                    Kg[ii][jj] += f * (p11 * gxi * gxj + p22 * gyi * gyj + p12 * (gxi * gyj + gyi * gxj) + gzi * gzj);
                }
            }
        }
    }
}

// geometric_stiffness_frame3d (FEMKernels.jl:7441-7471)
void frame3d_geometric(double L, double P, double kg[12][12]) {
    std::memset(kg, 0, sizeof(double) * 144);
    if (L < 1e-9 || std::fabs(P) < 1e-30) return;
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

// ---------------------------------------------------------------------------
// model-level assembly
// ---------------------------------------------------------------------------

struct Triplets {
    std::vector<int64_t> I, J;  // 0-based
    std::vector<double> V;
    // Rounding scale of each value (tests only; empty: |V|).  It differs from
    // |V| where the value is a product of a cancelling sum, e.g. a bar KG term
    // proportional to an axial force P that is a small difference of large
    // end displacements.
    std::vector<double> M;
};

const double *node_R_of(const jfg_model_desc *d, int64_t n, double tmp[9]) {
    if (d->node_R) return d->node_R + 9 * n;
    for (int i = 0; i < 9; ++i) tmp[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return tmp;
}

// Q4 frame (shell_element_frame_quad4 :diag mode, helpers.jl:1134-1193)
void q4_frame(const double *p1, const double *p2, const double *p3, const double *p4, double v1[3], double v2[3], double v3[3]) {
    double gxi[3], geta[3], v3r[3];
    for (int i = 0; i < 3; ++i) {
        gxi[i] = 0.25 * (-p1[i] + p2[i] + p3[i] - p4[i]);
        geta[i] = 0.25 * (-p1[i] - p2[i] + p3[i] + p4[i]);
    }
    cross3(gxi, geta, v3r);
    if (dot3(v3r, v3r) <= 1e-24) {
        double d13[3], d24[3];
        sub3(p3, p1, d13); sub3(p4, p2, d24);
        cross3(d13, d24, v3r);
    }
    normalize3(v3r, v3);
    double d13[3], d24[3], d13n[3], d24n[3], xr[3];
    sub3(p3, p1, d13); sub3(p4, p2, d24);
    normalize3(d13, d13n); normalize3(d24, d24n);
    for (int i = 0; i < 3; ++i) xr[i] = d13n[i] - d24n[i];
    if (dot3(xr, xr) < 1e-20)
        for (int i = 0; i < 3; ++i) xr[i] = d13n[i] + d24n[i];
    double xp[3], dv = dot3(xr, v3);
    for (int i = 0; i < 3; ++i) xp[i] = xr[i] - dv * v3[i];
    if (dot3(xp, xp) <= 1e-24) {
        double ga = dot3(geta, v3);
        for (int i = 0; i < 3; ++i) xp[i] = geta[i] - ga * v3[i];
        if (dot3(xp, xp) <= 1e-24) {
            double e[3];
            sub3(p2, p1, e);
            double ev = dot3(e, v3);
            for (int i = 0; i < 3; ++i) xp[i] = e[i] - ev * v3[i];
        }
    }
    normalize3(xp, v1);
    cross3(v3, v1, v2);
}

// flatness test of the K/KG loops (assembly.jl:2824-2840, :4817-4832)
bool q4_is_flat(const double *p1, const double *p2, const double *p3, const double *p4) {
    double d13[3], d24[3], n[3], c[3];
    sub3(p3, p1, d13); sub3(p4, p2, d24);
    cross3(d13, d24, n);
    double len = norm3(n);
    for (int i = 0; i < 3; ++i) c[i] = (p1[i] + p2[i] + p3[i] + p4[i]) / 4.0;
    double maxdev = 0.0;
    if (len > 1e-12) {
        double g[3] = {n[0] / len, n[1] / len, n[2] / len};
        const double *ps[4] = {p1, p2, p3, p4};
        for (int k = 0; k < 4; ++k) {
            double d[3];
            sub3(ps[k], c, d);
            maxdev = std::max(maxdev, std::fabs(dot3(d, g)));
        }
    }
    double L = std::max(norm3(d13), norm3(d24));
    return maxdev < 1e-6 * std::max(L, 1e-12);
}

void shell_constitutive(const double *pr, double Cm[3][3], double Cb[3][3], double Cs[2][2]) {
    double h = pr[0], E = pr[1], nu = pr[2], br = pr[4], tst = pr[5], Gs = pr[6];
    double cm = E * h / (1 - nu * nu);
    double cb = br * (E * h * h * h) / (12 * (1 - nu * nu));
    double base[3][3] = {{1.0, nu, 0.0}, {nu, 1.0, 0.0}, {0.0, 0.0, (1 - nu) / 2}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Cm[i][j] = cm * base[i][j]; Cb[i][j] = cb * base[i][j]; }
    double G = Gs;
    Cs[0][0] = tst * h * G; Cs[0][1] = 0.0; Cs[1][0] = 0.0; Cs[1][1] = tst * h * G;
    if (br <= 1e-12) { Cs[0][0] = Cs[0][1] = Cs[1][0] = Cs[1][1] = 0.0; }
}

// T' K T for a block-diagonal T built from 3x3 node blocks Q_k = Rel * node_R
void transform_sym(int nn, const double *Q /* nn*9 */, const double *K, double *out) {
    int n = 6 * nn;
    std::vector<double> T(n * n, 0.0), tmp(n * n, 0.0);
    for (int k = 0; k < nn; ++k)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                T[(6 * k + r) * n + 6 * k + c] = Q[9 * k + 3 * r + c];
                T[(6 * k + 3 + r) * n + 6 * k + 3 + c] = Q[9 * k + 3 * r + c];
            }
    mul(tmp.data(), K, T.data(), n, n, n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int l = 0; l < n; ++l) s += T[l * n + i] * tmp[l * n + j];
            out[i * n + j] = s;
        }
}

// ---------------------------------------------------------------------------
// Rounding scales of KG element values (tests only).  A KG term is a product
// of a membrane stress or a bar axial force, which the element forms from
// differences of nodal displacements.  Where that stress or force is small
// next to the displacement terms it is formed from, any two implementations
// (the reference's own included) round it differently by eps times those
// terms.  These functions carry the magnitudes of the terms, instead of the
// values, through the same products, giving each KG value's rounding scale.
// ---------------------------------------------------------------------------

// |Q|' K |Q| for the block-diagonal node rotations (K >= 0 entrywise).
void transform_sym_abs(int nn, const double *Q, const double *K, double *out) {
    int n = 6 * nn;
    std::vector<double> T(n * n, 0.0), tmp(n * n, 0.0);
    for (int k = 0; k < nn; ++k)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                T[(6 * k + r) * n + 6 * k + c] = std::fabs(Q[9 * k + 3 * r + c]);
                T[(6 * k + 3 + r) * n + 6 * k + 3 + c] = std::fabs(Q[9 * k + 3 * r + c]);
            }
    mul(tmp.data(), K, T.data(), n, n, n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int l = 0; l < n; ++l) s += T[l * n + i] * tmp[l * n + j];
            out[i * n + j] = s;
        }
}

// Scale of the local displacements u_loc = Q u_global: sum |Q_rl u_l|.
void local_u_scale(int nn, const int32_t *nd, const double *Q, const double *u, double *us) {
    for (int k = 0; k < nn; ++k) {
        const double *ug = u + 6 * (int64_t)nd[k];
        for (int dd = 0; dd < 3; ++dd) {
            double a = 0.0, b = 0.0;
            for (int l = 0; l < 3; ++l) {
                a += std::fabs(Q[9 * k + 3 * dd + l] * ug[l]);
                b += std::fabs(Q[9 * k + 3 * dd + l] * ug[3 + l]);
            }
            us[6 * k + dd] = a;
            us[6 * k + 3 + dd] = b;
        }
    }
}

// CQUAD4 KG (principal-transverse, incompatible membrane modes): the stress
// of every Gauss point over the magnitudes of its strain terms (B u and the
// incompatible modes B_i alpha, alpha = -K_bb^-1 K_ab' u), then both
// principal directions with |lambda| <= |sxx| + |syy| + 2 |sxy| and
// |cos|, |sin| <= 1 over the gradient vectors' magnitudes.  The direction
// itself, theta = atan2(2 sxy, sxx - syy) / 2, moves by the stress rounding
// over twice the deviatoric radius rad = |lambda_1 - lambda_2| / 2, and the
// transverse terms move with it (d/dtheta of a unit direction is bounded by
// the same gradient magnitudes): near an equibiaxial stress the reference's
// own KG is that ill-conditioned, so the scale grows as 1 / rad there.
// sig holds the Gauss-point stresses the element computed.
void q4_kg_scale(const double lc[4][2], const double us[24], const double Cm[3][3], double h, const double sig[4][3],
                 double M[24][24]) {
    std::memset(M, 0, sizeof(double) * 576);
    if (h < 1e-30) return;
    const double pt = 1.0 / std::sqrt(3.0);
    const double gp[4][2] = {{-pt, -pt}, {pt, -pt}, {pt, pt}, {-pt, pt}};
    double K_ab[24][4] = {}, K_bb[4][4] = {}, Bm[4][3][24] = {}, Bi[4][3][4] = {}, det[4];
    Jac js[4];
    for (int g = 0; g < 4; ++g) {
        double dNr[4], dNs[4];
        shape_derivs_quad(gp[g][0], gp[g][1], dNr, dNs);
        js[g] = jacobian(lc, dNr, dNs);
        det[g] = std::max(std::fabs(js[g].det), 1e-12);
        for (int k = 0; k < 4; ++k) {
            const double dx = js[g].iJ11 * dNr[k] + js[g].iJ12 * dNs[k], dy = js[g].iJ21 * dNr[k] + js[g].iJ22 * dNs[k];
            Bm[g][0][6 * k] = dx; Bm[g][1][6 * k + 1] = dy; Bm[g][2][6 * k] = dy; Bm[g][2][6 * k + 1] = dx;
        }
        const double r = gp[g][0], s = gp[g][1];
        const double d1x = js[g].iJ11 * (-2.0 * r), d1y = js[g].iJ21 * (-2.0 * r), d2x = js[g].iJ12 * (-2.0 * s),
                     d2y = js[g].iJ22 * (-2.0 * s);
        Bi[g][0][0] = d1x; Bi[g][2][0] = d1y; Bi[g][1][1] = d1y; Bi[g][2][1] = d1x;
        Bi[g][0][2] = d2x; Bi[g][2][2] = d2y; Bi[g][1][3] = d2y; Bi[g][2][3] = d2x;
        double CBi[12];
        mul(CBi, &Cm[0][0], &Bi[g][0][0], 3, 3, 4);
        mul_At_add(&K_ab[0][0], &Bm[g][0][0], CBi, 3, 24, 4, det[g]);
        mul_At_add(&K_bb[0][0], &Bi[g][0][0], CBi, 3, 4, 4, det[g]);
    }
    double Kbi[4][4], am[4], Amap[4][24];
    inv4(K_bb, Kbi);
    q4_incomp_map(lc, Cm, Amap);
    for (int l = 0; l < 4; ++l) {
        double r = 0.0;
        for (int m = 0; m < 4; ++m) {
            double t = 0.0;
            for (int i = 0; i < 24; ++i) t += std::fabs(K_ab[i][m]) * us[i];
            r += std::fabs(Kbi[l][m]) * t;
        }
        am[l] = r;
    }
    for (int g = 0; g < 4; ++g) {
        double em[3], sm[3];
        for (int c = 0; c < 3; ++c) {
            double t = 0.0;
            for (int i = 0; i < 24; ++i) t += std::fabs(Bm[g][c][i]) * us[i];
            for (int l = 0; l < 4; ++l) t += std::fabs(Bi[g][c][l]) * am[l];
            em[c] = t;
        }
        for (int c = 0; c < 3; ++c) sm[c] = (std::fabs(Cm[c][0]) * em[0] + std::fabs(Cm[c][1]) * em[1] + std::fabs(Cm[c][2]) * em[2]) / h;
        const double lam = sm[0] + sm[1] + 2.0 * sm[2];
        const double r = gp[g][0], s = gp[g][1];
        const double d1x = js[g].iJ11 * (-2.0 * r), d1y = js[g].iJ21 * (-2.0 * r), d2x = js[g].iJ12 * (-2.0 * s),
                     d2y = js[g].iJ22 * (-2.0 * s);
        double Gxy[24] = {}, Gz[24] = {};
        double dNr[4], dNs[4];
        shape_derivs_quad(r, s, dNr, dNs);
        for (int k = 0; k < 4; ++k) {
            const double dx = std::fabs(js[g].iJ11 * dNr[k] + js[g].iJ12 * dNs[k]),
                         dy = std::fabs(js[g].iJ21 * dNr[k] + js[g].iJ22 * dNs[k]);
            Gxy[6 * k] += dx + dy; Gxy[6 * k + 1] += dx + dy; Gz[6 * k + 2] = dx + dy;
        }
        for (int a = 0; a < 24; ++a)
            Gxy[a] += (std::fabs(d1x) + std::fabs(d1y)) * (std::fabs(Amap[0][a]) + std::fabs(Amap[1][a])) +
                      (std::fabs(d2x) + std::fabs(d2y)) * (std::fabs(Amap[2][a]) + std::fabs(Amap[3][a]));
        const double f = 2.0 * h * det[g] * lam;
        const double hd = 0.5 * (sig[g][0] - sig[g][1]), rad = std::sqrt(hd * hd + sig[g][2] * sig[g][2]);
        const double dth = lam / (2.0 * std::max(rad, 1e-30));  // rounding of theta, in units of eps
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j)
                M[i][j] += f * (Gxy[i] * Gxy[j] + Gz[i] * Gz[j]) + f * dth * (4.0 * Gxy[i] * Gxy[j] + 2.0 * Gz[i] * Gz[j]);
    }
}

struct Err { int code = 0; std::string msg; };

int check_predicates(const jfg_model_desc *d, std::string &msg) {
    if (d->param_snorm > 0.0) { msg = "PARAM,SNORM > 0 leaves the default branch (snorm.jl:72-83)"; return JFG_ERR_UNSUPPORTED; }
    for (int64_t e = 0; e < d->n_quad4; ++e) {
        const int32_t *n = d->quad4_nodes + 4 * e;
        if (!(d->quad4_prop[JFG_SHELL_PROP * e] > 0.0) || !(d->quad4_prop[JFG_SHELL_PROP * e + 1] > 0.0)) { msg = "shell thickness and E must be positive"; return JFG_ERR_INVALID; }
        for (int k = 0; k < 4; ++k)
            if (n[k] < 0 || n[k] >= d->n_nodes) { msg = "quad4 node index out of range"; return JFG_ERR_INVALID; }
        for (int a = 0; a < 4; ++a)
            for (int b = a + 1; b < 4; ++b)
                if (n[a] == n[b]) { msg = "CQUAD4 with a repeated node"; return JFG_ERR_INVALID; }
        if (!q4_is_flat(d->coords + 3 * n[0], d->coords + 3 * n[1], d->coords + 3 * n[2], d->coords + 3 * n[3])) {
            msg = "non-flat CQUAD4 (warp >= 1e-6 of the diagonal) leaves the flat default branch (assembly.jl:2824-2840)";
            return JFG_ERR_UNSUPPORTED;
        }
    }
    for (int64_t e = 0; e < d->n_tria3; ++e) {
        if (!(d->tria3_prop[JFG_SHELL_PROP * e] > 0.0) || !(d->tria3_prop[JFG_SHELL_PROP * e + 1] > 0.0)) { msg = "shell thickness and E must be positive"; return JFG_ERR_INVALID; }
        for (int k = 0; k < 3; ++k)
            if (d->tria3_nodes[3 * e + k] < 0 || d->tria3_nodes[3 * e + k] >= d->n_nodes) { msg = "tria3 node index out of range"; return JFG_ERR_INVALID; }
        const int32_t *tn = d->tria3_nodes + 3 * e;
        if (tn[0] == tn[1] || tn[0] == tn[2] || tn[1] == tn[2]) { msg = "CTRIA3 with a repeated node"; return JFG_ERR_INVALID; }
    }
    for (int64_t e = 0; e < d->n_bar; ++e) {
        for (int k = 0; k < 2; ++k)
            if (d->bar_nodes[2 * e + k] < 0 || d->bar_nodes[2 * e + k] >= d->n_nodes) { msg = "bar node index out of range"; return JFG_ERR_INVALID; }
        if (d->bar_pin && (d->bar_pin[2 * e] != 0 || d->bar_pin[2 * e + 1] != 0)) {
            msg = "CBAR pin flags PA/PB are outside the supported branch (helpers.jl:1630-1660)"; return JFG_ERR_UNSUPPORTED;
        }
    }
    return 0;
}

// Q4 and T3 geometry helpers shared by K and KG
void t3_frame(const double *p1, const double *p2, const double *p3, double v1[3], double v2[3], double v3[3]) {
    double e[3], f[3], c[3];
    sub3(p2, p1, e);
    normalize3(e, v1);
    sub3(p3, p1, f);
    cross3(v1, f, c);
    normalize3(c, v3);
    cross3(v3, v1, v2);
}

void node_blocks(const jfg_model_desc *d, const int32_t *nodes, int nn, const double v1[3], const double v2[3], const double v3[3], double *Q) {
    double Rel[9] = {v1[0], v1[1], v1[2], v2[0], v2[1], v2[2], v3[0], v3[1], v3[2]};
    for (int k = 0; k < nn; ++k) {
        double tmp[9];
        const double *R = node_R_of(d, nodes[k], tmp);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Q[9 * k + 3 * r + c] = Rel[3 * r] * R[c] + Rel[3 * r + 1] * R[3 + c] + Rel[3 * r + 2] * R[6 + c];
    }
}

// bar frame + T12 (assembly.jl:3961-4025)
bool bar_setup(const jfg_model_desc *d, int64_t e, double &L, double T12[12][12], bool &has_offset) {
    const int32_t *nd = d->bar_nodes + 2 * e;
    const double *pr = d->bar_prop + JFG_BAR_PROP * e;
    const double *p1 = d->coords + 3 * nd[0], *p2 = d->coords + 3 * nd[1];
    double wa[3] = {pr[12], pr[13], pr[14]}, wb[3] = {pr[15], pr[16], pr[17]};
    has_offset = dot3(wa, wa) > 1e-20 || dot3(wb, wb) > 1e-20;
    double a[3], b[3];
    for (int i = 0; i < 3; ++i) { a[i] = has_offset ? p1[i] + wa[i] : p1[i]; b[i] = has_offset ? p2[i] + wb[i] : p2[i]; }
    double dd[3];
    sub3(b, a, dd);
    L = norm3(dd);
    if (L < 1e-9) return false;
    double vx[3], vref[3] = {pr[9], pr[10], pr[11]}, vz[3], vy[3], t[3];
    normalize3(dd, vx);
    if (norm3(vref) < 1e-6) {
        vref[0] = 0.0; vref[1] = 0.0; vref[2] = 1.0;
        if (std::fabs(dot3(vx, vref)) > 0.9) { vref[0] = 0.0; vref[1] = 1.0; vref[2] = 0.0; }
    }
    cross3(vx, vref, t);
    normalize3(t, vz);
    cross3(vz, vx, vy);
    double Rel[3][3] = {{vx[0], vx[1], vx[2]}, {vy[0], vy[1], vy[2]}, {vz[0], vz[1], vz[2]}};
    std::memset(T12, 0, sizeof(double) * 144);
    for (int k = 0; k < 2; ++k) {
        double tmp[9];
        const double *R = node_R_of(d, nd[k], tmp);
        double TR[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) TR[r][c] = Rel[r][0] * R[c] + Rel[r][1] * R[3 + c] + Rel[r][2] * R[6 + c];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) { T12[6 * k + r][6 * k + c] = TR[r][c]; T12[6 * k + 3 + r][6 * k + 3 + c] = TR[r][c]; }
        if (has_offset) {
            const double *w = k == 0 ? wa : wb;
            double S[3][3] = {{0.0, -w[2], w[1]}, {w[2], 0.0, -w[0]}, {-w[1], w[0], 0.0}};
            double RS[3][3];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) RS[r][c] = Rel[r][0] * S[0][c] + Rel[r][1] * S[1][c] + Rel[r][2] * S[2][c];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) T12[6 * k + r][6 * k + 3 + c] = -(RS[r][0] * R[c] + RS[r][1] * R[3 + c] + RS[r][2] * R[6 + c]);
        }
    }
    return true;
}

void bar_section(const double *pr, double &A, double &Iy, double &Iz, double &I12, double &J, double &E, double &G, double &Asy, double &Asz) {
    A = pr[0];
    Iy = pr[2]; Iz = pr[1];
    if (Iy == 0.0) Iy = Iz;
    if (Iz == 0.0) Iz = Iy;
    I12 = pr[3]; J = pr[4];
    double K1 = pr[5], K2 = pr[6];
    E = pr[7]; G = pr[8];
    Asy = K1 > 0.0 ? K1 * A : INFINITY;
    Asz = K2 > 0.0 ? K2 * A : INFINITY;
}

// RBE2 dependent map (constraints.jl:7-74)
std::map<int64_t, std::vector<std::pair<int64_t, double>>> rbe2_map(const jfg_model_desc *d) {
    std::map<int64_t, std::vector<std::pair<int64_t, double>>> mp;
    for (int64_t r = 0; r < d->n_rbe2; ++r) {
        int64_t gm = d->rbe2_master[r];
        const double *pm = d->coords + 3 * gm;
        double tm[9];
        const double *Rm = node_R_of(d, gm, tm);
        for (int64_t s = d->rbe2_slave_ptr[r]; s < d->rbe2_slave_ptr[r + 1]; ++s) {
            int64_t gs = d->rbe2_slaves[s];
            const double *ps = d->coords + 3 * gs;
            double dx = ps[0] - pm[0], dy = ps[1] - pm[1], dz = ps[2] - pm[2];
            double ts[9];
            const double *Rs = node_R_of(d, gs, ts);
            double comp[3][3], O[3][3] = {{0.0, dz, -dy}, {-dz, 0.0, dx}, {dy, -dx, 0.0}}, RsO[3][3], off[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) comp[i][j] = Rs[i] * Rm[j] + Rs[3 + i] * Rm[3 + j] + Rs[6 + i] * Rm[6 + j];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) RsO[i][j] = Rs[i] * O[0][j] + Rs[3 + i] * O[1][j] + Rs[6 + i] * O[2][j];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) off[i][j] = RsO[i][0] * Rm[j] + RsO[i][1] * Rm[3 + j] + RsO[i][2] * Rm[6 + j];
            for (int c = 1; c <= 6; ++c) {
                if (!(d->rbe2_cm[r] & (1 << (c - 1)))) continue;
                double row[6];
                if (c <= 3) {
                    for (int j = 0; j < 3; ++j) { row[j] = comp[c - 1][j]; row[3 + j] = off[c - 1][j]; }
                } else {
                    for (int j = 0; j < 3; ++j) { row[j] = 0.0; row[3 + j] = comp[c - 4][j]; }
                }
                std::vector<std::pair<int64_t, double>> pairs;
                for (int j = 0; j < 6; ++j)
                    if (std::fabs(row[j]) > 1e-15) pairs.push_back({6 * gm + j, row[j]});
                if (!pairs.empty()) mp[6 * gs + (c - 1)] = pairs;
            }
        }
    }
    return mp;
}

// Triplet redistribution (constraints.jl:329-361) followed by
// SparseArrays.sparse(I, J, V, n, n) to 1-based CSC.
//
// sparse() is restated from SparseArrays' published algorithm (sparse! in
// SparseArrays 1.12): (1) a counting sort of the triplets into rows, keeping
// input order inside each row; (2) per row, every repeated column is merged
// into its first occurrence, summing left to right in input order (the
// combine = + fold, explicit zeros kept); (3) the row-compressed result is
// transposed into CSC, which leaves each column's rows ascending.  It is
// O(triplets + n) and serial, like the reference's.  The redistribution is
// applied on the fly in both counting passes, in the reference's emission
// order (images of a dependent dof in the order of its constraint row), so
// the redistributed triplet list is never materialised.
//
// abs_sums (optional) receives, per stored entry, the same fold over the
// terms' rounding scales (|v|, or t.M): the scale of the entry's rounding
// in any summation order.  Only the tests use it.
void constrain_and_csc(const jfg_model_desc *d, Triplets &t, std::vector<int64_t> &colptr, std::vector<int64_t> &rowval,
                       std::vector<double> &nzval, std::vector<double> *abs_sums = nullptr) {
    auto mp = rbe2_map(d);
    const int64_t ndof = 6 * d->n_nodes;
    std::vector<const std::vector<std::pair<int64_t, double>> *> dep(ndof, nullptr);
    for (auto &kv : mp) dep[kv.first] = &kv.second;
    const size_t n_in = t.V.size();
    // f(i, j, v, mag) for every triplet that input k becomes, in emission
    // order; mag is the rounding scale of v (|v| unless t.M says otherwise)
    const bool has_m = !t.M.empty();
    auto emit = [&](size_t k, auto &&f) {
        const int64_t i = t.I[k], j = t.J[k];
        const double v = t.V[k], mg = has_m ? t.M[k] : std::fabs(v);
        const auto *di = dep[i], *dj = dep[j];
        if (!di && !dj) f(i, j, v, mg);
        else if (di && !dj) { for (auto &p : *di) f(p.first, j, v * p.second, mg * std::fabs(p.second)); }
        else if (!di && dj) { for (auto &p : *dj) f(i, p.first, v * p.second, mg * std::fabs(p.second)); }
        else {
            for (auto &a : *di)
                for (auto &b : *dj) f(a.first, b.first, v * a.second * b.second, mg * std::fabs(a.second * b.second));
        }
    };
    // (1) counting sort into rows
    std::vector<int64_t> row_at(ndof + 1, 0);
    for (size_t k = 0; k < n_in; ++k) emit(k, [&](int64_t i, int64_t, double, double) { ++row_at[i + 1]; });
    for (int64_t i = 0; i < ndof; ++i) row_at[i + 1] += row_at[i];
    const int64_t n_trip = row_at[ndof];
    std::vector<int32_t> ccol(n_trip);
    std::vector<double> cval(n_trip), cabs(abs_sums ? n_trip : 0);
    {
        std::vector<int64_t> fill(row_at.begin(), row_at.end() - 1);
        for (size_t k = 0; k < n_in; ++k)
            emit(k, [&](int64_t i, int64_t j, double v, double mg) {
                const int64_t q = fill[i]++;
                ccol[q] = (int32_t)j;
                cval[q] = v;
                if (abs_sums) cabs[q] = mg;
            });
    }
    // (2) merge repeated columns per row into their first occurrence, in order
    std::vector<int64_t> last(ndof, -1), crow(ndof + 1, 0);
    int64_t w = 0;
    for (int64_t i = 0; i < ndof; ++i) {
        crow[i] = w;
        for (int64_t q = row_at[i]; q < row_at[i + 1]; ++q) {
            const int32_t j = ccol[q];
            if (last[j] < crow[i]) {
                last[j] = w;
                ccol[w] = j;
                cval[w] = cval[q];
                if (abs_sums) cabs[w] = cabs[q];
                ++w;
            } else {
                cval[last[j]] += cval[q];
                if (abs_sums) cabs[last[j]] += cabs[q];
            }
        }
    }
    crow[ndof] = w;
    // (3) transpose to CSC (rows ascending within each column), 1-based
    colptr.assign(ndof + 1, 0);
    for (int64_t q = 0; q < w; ++q) ++colptr[ccol[q] + 1];
    for (int64_t c = 0; c < ndof; ++c) colptr[c + 1] += colptr[c];
    rowval.assign(w, 0);
    nzval.assign(w, 0.0);
    if (abs_sums) abs_sums->assign(w, 0.0);
    {
        std::vector<int64_t> next(colptr.begin(), colptr.end() - 1);
        for (int64_t i = 0; i < ndof; ++i)
            for (int64_t q = crow[i]; q < crow[i + 1]; ++q) {
                const int64_t r = next[ccol[q]]++;
                rowval[r] = i + 1;
                nzval[r] = cval[q];
                if (abs_sums) (*abs_sums)[r] = cabs[q];
            }
    }
    for (auto &c : colptr) c += 1;
}

}  // namespace

// ---------------------------------------------------------------------------
// shell-thickness sensitivity element (dKdx.jl:218-250)
// ---------------------------------------------------------------------------

// stiffness_quad4_generic (FEMKernels.jl:1473-1490) over
// stiffness_quad4_default_generic (:1496-1656), the element that
// _shell_thickness_dKe_forward_ad differentiates: bend_ratio 1, ts_t 5/6,
// k6rot 100, G = E / 2(1 + nu) (drill G_ref too), membrane with Wilson
// incompatible modes at the Gauss-point Jacobian (no bending modes), bending
// without the twist row, and transverse shear from the four tying points
// (0, -+1), (-+1, 0) scaled by phi2 = min(1, 10 h^2 / max(4 |det Jc|, 1e-30))
// (PHI2_ALPHA = 10, :10).  The parts are kept apart so that
//   K      = Km + Kb + Kd + Ks - Kc
//   dK/dh  = (Km + Kd - Kc + 3 Kb + s Ks) / h,   s = 3 while phi2 < 1, else 1,
// which is what forward-mode AD of the reference returns: Cm, K_ab, K_bb and
// the drill scale are linear in h, Cb cubic, and Cs linear times phi2 (h^2 on
// the unsaturated branch ForwardDiff takes, constant on the saturated one).
struct Q4GenericParts {
    double Km[24][24], Kb[24][24], Kd[24][24], Ks[24][24], Kc[24][24];
    bool phi2_saturated;
};

void q4_generic_parts(const double lc[4][2], double E, double nu, double h, Q4GenericParts &P) {
    std::memset(&P, 0, sizeof(P));
    const double cm = E * h / (1 - nu * nu), cb = 1.0 * (E * h * h * h) / (12 * (1 - nu * nu));
    const double base[3][3] = {{1.0, nu, 0.0}, {nu, 1.0, 0.0}, {0.0, 0.0, (1 - nu) / 2}};
    double Cm[3][3], Cb[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Cm[i][j] = cm * base[i][j]; Cb[i][j] = cb * base[i][j]; }
    const double G = E / (2 * (1 + nu));
    const double cs = (5.0 / 6.0) * G * h;
    // tying-point rows (w, theta_x, theta_y of each node), :1510-1538
    double Bs_tp[4][24] = {};
    const double tp[4][2] = {{0.0, -1.0}, {0.0, 1.0}, {-1.0, 0.0}, {1.0, 0.0}};
    for (int t = 0; t < 4; ++t) {
        double dNr[4], dNs[4];
        shape_derivs_quad(tp[t][0], tp[t][1], dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        const double xi = tp[t][0], eta = tp[t][1];
        const double N[4] = {0.25 * (1.0 - xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 + eta),
                             0.25 * (1.0 - xi) * (1.0 + eta)};
        for (int k = 0; k < 4; ++k) {
            if (t < 2) { Bs_tp[t][6 * k + 2] = dNr[k]; Bs_tp[t][6 * k + 3] = -j.J12 * N[k]; Bs_tp[t][6 * k + 4] = j.J11 * N[k]; }
            else { Bs_tp[t][6 * k + 2] = dNs[k]; Bs_tp[t][6 * k + 3] = -j.J22 * N[k]; Bs_tp[t][6 * k + 4] = j.J21 * N[k]; }
        }
    }
    const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25}, dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
    Jac jc = jacobian(lc, dNr_c, dNs_c);
    const double L_char_sq = std::max(4.0 * std::fabs(jc.det), 1e-30);
    const double phi2_trial = 10.0 * h * h / L_char_sq;
    P.phi2_saturated = !(phi2_trial < 1.0);
    const double phi2 = P.phi2_saturated ? 1.0 : phi2_trial;
    const double alpha_drill = (100.0 / 1e5) * G * h;
    double K_ab[24][4] = {}, K_bb[4][4] = {};
    const double pt = 1.0 / std::sqrt(3.0);
    const double gp[4][2] = {{-pt, -pt}, {pt, -pt}, {pt, pt}, {-pt, pt}};
    for (int g = 0; g < 4; ++g) {
        const double r = gp[g][0], s = gp[g][1];
        double dNr[4], dNs[4];
        shape_derivs_quad(r, s, dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        double absdet = std::fabs(j.det);
        if (absdet < 1e-12) absdet = 1e-12;
        double Bm[3][24] = {}, Bb[3][24] = {}, Bd[1][24] = {}, Bi[3][4] = {};
        for (int k = 0; k < 4; ++k) {
            const double dx = j.iJ11 * dNr[k] + j.iJ12 * dNs[k], dy = j.iJ21 * dNr[k] + j.iJ22 * dNs[k];
            const int idx = 6 * k;
            const double Nk = 0.25 * (1 + ((k == 1 || k == 2) ? r : -r)) * (1 + (k >= 2 ? s : -s));
            Bm[0][idx] = dx; Bm[1][idx + 1] = dy; Bm[2][idx] = dy; Bm[2][idx + 1] = dx;
            Bb[0][idx + 4] = dx; Bb[1][idx + 3] = -dy; Bb[2][idx + 4] = dy; Bb[2][idx + 3] = -dx;
            Bd[0][idx] = 0.5 * dy; Bd[0][idx + 1] = -0.5 * dx; Bd[0][idx + 5] = Nk;
        }
        const double d1x = j.iJ11 * (-2.0 * r), d1y = j.iJ21 * (-2.0 * r), d2x = j.iJ12 * (-2.0 * s), d2y = j.iJ22 * (-2.0 * s);
        Bi[0][0] = d1x; Bi[2][0] = d1y; Bi[1][1] = d1y; Bi[2][1] = d1x;
        Bi[0][2] = d2x; Bi[2][2] = d2y; Bi[1][3] = d2y; Bi[2][3] = d2x;
        double t3x24[3 * 24], t3x4[3 * 4];
        mul(t3x24, &Cm[0][0], &Bm[0][0], 3, 3, 24);
        mul_At_add(&P.Km[0][0], &Bm[0][0], t3x24, 3, 24, 24, absdet);
        mul(t3x24, &Cb[0][0], &Bb[0][0], 3, 3, 24);
        mul_At_add(&P.Kb[0][0], &Bb[0][0], t3x24, 3, 24, 24, absdet);
        mul_At_add(&P.Kd[0][0], &Bd[0][0], &Bd[0][0], 1, 24, 24, absdet * alpha_drill);
        // covariant shear interpolation and Cs_cov = phi2 invJ' Cs invJ (:1620-1634)
        const double wem = 0.5 * (1.0 - s), wep = 0.5 * (1.0 + s), wxm = 0.5 * (1.0 - r), wxp = 0.5 * (1.0 + r);
        double Bs[2][24];
        for (int c = 0; c < 24; ++c) {
            Bs[0][c] = wem * Bs_tp[0][c] + wep * Bs_tp[1][c];
            Bs[1][c] = wxm * Bs_tp[2][c] + wxp * Bs_tp[3][c];
        }
        const double iJ[2][2] = {{j.iJ11, j.iJ12}, {j.iJ21, j.iJ22}};
        double Csc[2][2];
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) Csc[a][b] = phi2 * cs * (iJ[0][a] * iJ[0][b] + iJ[1][a] * iJ[1][b]);
        double t2x24[2 * 24];
        mul(t2x24, &Csc[0][0], &Bs[0][0], 2, 2, 24);
        mul_At_add(&P.Ks[0][0], &Bs[0][0], t2x24, 2, 24, 24, absdet);
        mul(t3x4, &Cm[0][0], &Bi[0][0], 3, 3, 4);
        mul_At_add(&K_ab[0][0], &Bm[0][0], t3x4, 3, 24, 4, absdet);
        mul_At_add(&K_bb[0][0], &Bi[0][0], t3x4, 3, 4, 4, absdet);
    }
    double kbbmax = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int c = 0; c < 4; ++c) kbbmax = std::max(kbbmax, std::fabs(K_bb[i][c]));
    if (kbbmax > 0.0) {
        // K_ab (K_bb \ K_ab')
        double A[16], X[4 * 24];
        for (int i = 0; i < 4; ++i)
            for (int c = 0; c < 4; ++c) A[4 * i + c] = K_bb[i][c];
        for (int l = 0; l < 4; ++l)
            for (int c = 0; c < 24; ++c) X[24 * l + c] = K_ab[c][l];
        lu_solve(4, 24, A, X);
        for (int i = 0; i < 24; ++i)
            for (int c = 0; c < 24; ++c) {
                double sm = 0.0;
                for (int l = 0; l < 4; ++l) sm += K_ab[i][l] * X[24 * l + c];
                P.Kc[i][c] = sm;
            }
    }
}

void q4_generic(const double lc[4][2], double E, double nu, double h, double Ke[24][24], double dKe[24][24]) {
    static thread_local Q4GenericParts P;
    q4_generic_parts(lc, E, nu, h, P);
    const double sfac = P.phi2_saturated ? 1.0 : 3.0;
    for (int i = 0; i < 24; ++i)
        for (int c = 0; c < 24; ++c) {
            if (Ke) Ke[i][c] = P.Km[i][c] + P.Kb[i][c] + P.Kd[i][c] + P.Ks[i][c] - P.Kc[i][c];
            if (dKe) dKe[i][c] = (P.Km[i][c] + P.Kd[i][c] - P.Kc[i][c] + 3.0 * P.Kb[i][c] + sfac * P.Ks[i][c]) / h;
        }
}

// stiffness_tria3_generic (FEMKernels.jl:7113-7123): the assembly's CTRIA3
// with bend_ratio 1, ts_t 5/6, k6rot 100 and G = E / 2(1 + nu).
void t3_generic(const double lc[3][2], double E, double nu, double h, double Ke[18][18]) {
    const double G = E / (2 * (1 + nu));
    const double base[3][3] = {{1.0, nu, 0.0}, {nu, 1.0, 0.0}, {0.0, 0.0, (1 - nu) / 2}};
    double Dm[3][3], Db[3][3], Ds[2][2] = {{(5.0 / 6.0) * G * h, 0.0}, {0.0, (5.0 / 6.0) * G * h}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            Dm[i][j] = (E * h / (1 - nu * nu)) * base[i][j];
            Db[i][j] = 1.0 * (E * h * h * h / (12 * (1 - nu * nu))) * base[i][j];
        }
    t3_stiffness(lc, Dm, Db, Ds, h, G, 1.0, 100.0, Ke);
}

// dK/dh of the CTRIA3 by forward-mode differentiation, as the reference's
// _shell_thickness_dKe_forward_ad does (dKdx.jl:219-228): the same element
// evaluated on a dual thickness h + eps.  Exact up to rounding, pivots and
// branches chosen on the values like ForwardDiff's.
void t3_generic_dkdh(const double lc[3][2], double E, double nu, double h, double dKe[18][18]) {
    const double G = E / (2 * (1 + nu));
    const double base[3][3] = {{1.0, nu, 0.0}, {nu, 1.0, 0.0}, {0.0, 0.0, (1 - nu) / 2}};
    const Dual hd(h, 1.0);
    Dual Dm[3][3], Db[3][3], Ds[2][2];
    const Dual cm = E * hd / (1 - nu * nu), cb = 1.0 * (E * hd * hd * hd / (12 * (1 - nu * nu)));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Dm[i][j] = cm * base[i][j]; Db[i][j] = cb * base[i][j]; }
    Ds[0][0] = Ds[1][1] = (5.0 / 6.0) * G * hd;
    Ds[0][1] = Ds[1][0] = 0.0;
    static thread_local Dual K[18][18];
    t3_stiffness(lc, Dm, Db, Ds, hd, Dual(G), 1.0, 100.0, K);
    for (int i = 0; i < 18; ++i)
        for (int c = 0; c < 18; ++c) dKe[i][c] = K[i][c].d;
}

// Shell element setup of _shell_elem_local_data (dKdx.jl:128-176): frame
// (shell_element_frame_fast: the :diag quad frame, the edge frame for a
// triangle), centroid-relative local coordinates, node blocks Rel * node_R.
void shell_setup(const jfg_model_desc *d, const int32_t *nd, int nn, double lc[4][2], double *Q) {
    const double *p[4];
    for (int k = 0; k < nn; ++k) p[k] = d->coords + 3 * (int64_t)nd[k];
    double v1[3], v2[3], v3[3];
    if (nn == 4) q4_frame(p[0], p[1], p[2], p[3], v1, v2, v3);
    else t3_frame(p[0], p[1], p[2], v1, v2, v3);
    double c[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < nn; ++k)
        for (int i = 0; i < 3; ++i) c[i] += p[k][i];
    for (int i = 0; i < 3; ++i) c[i] /= nn;
    for (int k = 0; k < nn; ++k) {
        double dd[3];
        sub3(p[k], c, dd);
        lc[k][0] = dot3(dd, v1); lc[k][1] = dot3(dd, v2);
    }
    node_blocks(d, nd, nn, v1, v2, v3, Q);
}

// x_local = T x_elem (translations and rotations of node k by Q_k).
void to_local(int nn, const double *Q, const double *xg, const int32_t *nd, double *xl) {
    for (int k = 0; k < nn; ++k)
        for (int half = 0; half < 2; ++half)
            for (int r = 0; r < 3; ++r) {
                double s = 0.0;
                for (int c = 0; c < 3; ++c) s += Q[9 * k + 3 * r + c] * xg[6 * (int64_t)nd[k] + 3 * half + c];
                xl[6 * k + 3 * half + r] = s;
            }
}

// ---------------------------------------------------------------------------
// SOL 101 output recovery (stress_recovery.jl:163-593), default branch:
// isotropic PSHELL/MAT1, no SNORM normals, no curvature membrane (scale 0),
// Wilson modes with each Gauss point's own Jacobian, frame mode :diag.
// ---------------------------------------------------------------------------

// The Gauss-point loops shared by stress_strain_quad4 (FEMKernels.jl:6003-6195)
// and quad4_bilinear_corner_forces (:6197-6338): membrane strain Bm u + Bi alpha
// with alpha = -(K_bb \ K_ab' u), curvature Bb u, and the clamped |det J|.
// Returns false where the reference's LU of K_bb raises (exactly singular).
bool q4_gp_fields(const double lc[4][2], const double u[24], const double Cm[3][3], double eps[4][3], double kap[4][3],
                  double wdet[4]) {
    const double pt = 1.0 / std::sqrt(3.0);
    const double gp[4][2] = {{-pt, -pt}, {pt, -pt}, {pt, pt}, {-pt, pt}};
    double K_ab[24][4] = {}, K_bb[4][4] = {};
    double Bm_g[4][3][24] = {}, Bb_g[4][3][24] = {}, Bi_g[4][3][4] = {};
    for (int g = 0; g < 4; ++g) {
        double r = gp[g][0], s = gp[g][1];
        double dNr[4], dNs[4];
        shape_derivs_quad(r, s, dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        double detg = std::fabs(j.det);
        if (detg < 1e-12) detg = 1e-12;
        wdet[g] = detg;
        for (int k = 0; k < 4; ++k) {
            double dx = j.iJ11 * dNr[k] + j.iJ12 * dNs[k];
            double dy = j.iJ21 * dNr[k] + j.iJ22 * dNs[k];
            Bm_g[g][0][6 * k] = dx; Bm_g[g][1][6 * k + 1] = dy; Bm_g[g][2][6 * k] = dy; Bm_g[g][2][6 * k + 1] = dx;
            Bb_g[g][0][6 * k + 4] = dx; Bb_g[g][1][6 * k + 3] = -dy;
            Bb_g[g][2][6 * k + 4] = dy; Bb_g[g][2][6 * k + 3] = -dx;
        }
        // fill_quad4_membrane_incompatible_B! (FEMKernels.jl:1831-1857)
        double d1x = j.iJ11 * (-2.0 * r), d1y = j.iJ21 * (-2.0 * r), d2x = j.iJ12 * (-2.0 * s), d2y = j.iJ22 * (-2.0 * s);
        Bi_g[g][0][0] = d1x; Bi_g[g][2][0] = d1y; Bi_g[g][1][1] = d1y; Bi_g[g][2][1] = d1x;
        Bi_g[g][0][2] = d2x; Bi_g[g][2][2] = d2y; Bi_g[g][1][3] = d2y; Bi_g[g][2][3] = d2x;
        double CBi[12];
        mul(CBi, &Cm[0][0], &Bi_g[g][0][0], 3, 3, 4);
        mul_At_add(&K_ab[0][0], &Bm_g[g][0][0], CBi, 3, 24, 4, detg);
        mul_At_add(&K_bb[0][0], &Bi_g[g][0][0], CBi, 3, 4, 4, detg);
    }
    double rhs[4], A[16];
    for (int l = 0; l < 4; ++l) {
        double s = 0.0;
        for (int i = 0; i < 24; ++i) s += K_ab[i][l] * u[i];
        rhs[l] = s;
    }
    for (int i = 0; i < 4; ++i)
        for (int jj = 0; jj < 4; ++jj) A[i * 4 + jj] = K_bb[i][jj];
    if (!lu_solve(4, 1, A, rhs)) return false;
    for (int g = 0; g < 4; ++g)
        for (int c = 0; c < 3; ++c) {
            double se = 0.0, sk = 0.0;
            for (int i = 0; i < 24; ++i) { se += Bm_g[g][c][i] * u[i]; sk += Bb_g[g][c][i] * u[i]; }
            for (int l = 0; l < 4; ++l) se += Bi_g[g][c][l] * (-rhs[l]);
            eps[g][c] = se;
            kap[g][c] = sk;
        }
    return true;
}

// quad4_mitc4_center_shear_resultant (FEMKernels.jl:5927-6001) with
// PHI2_ALPHA = 10 (FEMKernels.jl:10) and ts_t = 5/6.
void q4_mitc4_center_shear(const double lc[4][2], const double u[24], double G, double h, double Q[2]) {
    const double tp[4][2] = {{0.0, -1.0}, {0.0, 1.0}, {-1.0, 0.0}, {1.0, 0.0}};
    double Bs[4][24] = {};
    for (int t = 0; t < 4; ++t) {
        double xi = tp[t][0], eta = tp[t][1];
        double dNr[4], dNs[4];
        shape_derivs_quad(xi, eta, dNr, dNs);
        Jac j = jacobian(lc, dNr, dNs);
        double Nt[4] = {0.25 * (1 - xi) * (1 - eta), 0.25 * (1 + xi) * (1 - eta), 0.25 * (1 + xi) * (1 + eta),
                        0.25 * (1 - xi) * (1 + eta)};
        for (int k = 0; k < 4; ++k) {
            if (t < 2) { Bs[t][6 * k + 2] = dNr[k]; Bs[t][6 * k + 3] = -j.J12 * Nt[k]; Bs[t][6 * k + 4] = j.J11 * Nt[k]; }
            else { Bs[t][6 * k + 2] = dNs[k]; Bs[t][6 * k + 3] = -j.J22 * Nt[k]; Bs[t][6 * k + 4] = j.J21 * Nt[k]; }
        }
    }
    double dNr[4], dNs[4];
    shape_derivs_quad(0.0, 0.0, dNr, dNs);
    Jac c = jacobian(lc, dNr, dNs);
    double absdet = std::max(std::fabs(c.det), 1e-30);
    double gam[2] = {0.0, 0.0};
    for (int jx = 0; jx < 24; ++jx) {
        gam[0] += 0.5 * (Bs[0][jx] + Bs[1][jx]) * u[jx];
        gam[1] += 0.5 * (Bs[2][jx] + Bs[3][jx]) * u[jx];
    }
    double phi2 = std::min(1.0, 10.0 * h * h / std::max(4.0 * absdet, 1e-30));
    double k = 5.0 / 6.0 * G * h;
    double t11 = k * c.iJ11, t12 = k * c.iJ12, t21 = k * c.iJ21, t22 = k * c.iJ22;
    double M11 = c.iJ11 * t11 + c.iJ21 * t21, M12 = c.iJ11 * t12 + c.iJ21 * t22;
    double M21 = c.iJ12 * t11 + c.iJ22 * t21, M22 = c.iJ12 * t12 + c.iJ22 * t22;
    double q1 = phi2 * (M11 * gam[0] + M12 * gam[1]), q2 = phi2 * (M21 * gam[0] + M22 * gam[1]);
    Q[0] = c.J11 * q1 + c.J21 * q2;
    Q[1] = c.J12 * q1 + c.J22 * q2;
}

inline void plane_stress_D(double E, double nu, double D[3][3]) {
    double c = E / (1 - nu * nu);
    double b[3][3] = {{1.0, nu, 0.0}, {nu, 1.0, 0.0}, {0.0, 0.0, (1 - nu) / 2}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[i][j] = c * b[i][j];
}
inline void mv3(const double A[3][3], const double x[3], double y[3]) {
    for (int i = 0; i < 3; ++i) y[i] = A[i][0] * x[0] + A[i][1] * x[1] + A[i][2] * x[2];
}

// One element's recovered quantities (the record layout of JFG_SHELL_REC).
struct ShellRec {
    double N[3] = {}, M[3] = {}, Q[2] = {}, sz1[3] = {}, sz2[3] = {}, ez1[3] = {}, ez2[3] = {};
    double Nc[4][3] = {}, Mc[4][3] = {};
    bool ok = true;
};

// stress_strain_quad4 (for_kg = false), returning also the Gauss fields for
// the bilinear corner forces.
bool q4_stress_strain(const double lc[4][2], const double u[24], double E, double nu, double h, double br, ShellRec &R,
                      double eps[4][3], double kap[4][3]) {
    double D[3][3], Cm[3][3];
    plane_stress_D(E, nu, D);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Cm[i][j] = D[i][j] * h;
    double dNr[4], dNs[4];
    shape_derivs_quad(0.0, 0.0, dNr, dNs);
    if (jacobian(lc, dNr, dNs).det == 0.0) return false;  // inv(J) at the centre raises
    double wdet[4];
    if (!q4_gp_fields(lc, u, Cm, eps, kap, wdet)) return false;
    double ea[3] = {0, 0, 0}, ka[3] = {0, 0, 0}, area = 0.0;
    for (int g = 0; g < 4; ++g) {
        for (int c = 0; c < 3; ++c) { ea[c] += eps[g][c] * wdet[g]; ka[c] += kap[g][c] * wdet[g]; }
        area += wdet[g];
    }
    for (int c = 0; c < 3; ++c) { ea[c] /= area; ka[c] /= area; }
    mv3(Cm, ea, R.N);
    double Dk[3];
    mv3(D, ka, Dk);
    for (int c = 0; c < 3; ++c) R.M[c] = -br * Dk[c] * (h * h * h / 12.0);
    double G = E / (2 * (1 + nu));
    if (br <= 1e-12) R.Q[0] = R.Q[1] = 0.0;
    else q4_mitc4_center_shear(lc, u, G, h, R.Q);
    for (int c = 0; c < 3; ++c) { R.ez1[c] = ea[c] + (-h / 2.0) * ka[c]; R.ez2[c] = ea[c] + (h / 2.0) * ka[c]; }
    mv3(D, R.ez1, R.sz1);
    mv3(D, R.ez2, R.sz2);
    return true;
}

// quad4_bilinear_corner_forces: Gauss values N = Cm eps, M = -Cb kappa
// extrapolated to the corners (interp_2x2_gauss_sigma, FEMKernels.jl:5210-5227).
void q4_corner_forces(double E, double nu, double h, double br, const double eps[4][3], const double kap[4][3],
                      double Nc[4][3], double Mc[4][3]) {
    double D[3][3], Cm[3][3], Cb[3][3];
    plane_stress_D(E, nu, D);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Cm[i][j] = D[i][j] * h; Cb[i][j] = br * D[i][j] * (h * h * h / 12.0); }
    double Ng[4][3], Mg[4][3];
    for (int g = 0; g < 4; ++g) {
        mv3(Cm, eps[g], Ng[g]);
        double t[3];
        mv3(Cb, kap[g], t);
        for (int c = 0; c < 3; ++c) Mg[g][c] = -t[c];
    }
    const double pt = 1.0 / std::sqrt(3.0);
    const double cp[4][2] = {{-1.0, -1.0}, {1.0, -1.0}, {1.0, 1.0}, {-1.0, 1.0}};
    for (int i = 0; i < 4; ++i) {
        double xi = cp[i][0], eta = cp[i][1];
        double lx1 = (pt - xi) / (2.0 * pt), lx2 = (xi + pt) / (2.0 * pt), ly1 = (pt - eta) / (2.0 * pt), ly2 = (eta + pt) / (2.0 * pt);
        double w[4] = {lx1 * ly1, lx2 * ly1, lx2 * ly2, lx1 * ly2};
        for (int c = 0; c < 3; ++c) {
            Nc[i][c] = w[0] * Ng[0][c] + w[1] * Ng[1][c] + w[2] * Ng[2][c] + w[3] * Ng[3][c];
            Mc[i][c] = w[0] * Mg[0][c] + w[1] * Mg[1][c] + w[2] * Mg[2][c] + w[3] * Mg[3][c];
        }
    }
}

// _quad4_equilibrium_shear_from_bending + _quad4_blend_recovered_shear
// (stress_recovery.jl:88-130).
void q4_equilibrium_blend(const double lc[4][2], const double Mc[4][3], double Q[2]) {
    const double dNr[4] = {-0.25, 0.25, 0.25, -0.25}, dNs[4] = {-0.25, -0.25, 0.25, 0.25};
    double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
    for (int k = 0; k < 4; ++k) { J11 += dNr[k] * lc[k][0]; J12 += dNr[k] * lc[k][1]; J21 += dNs[k] * lc[k][0]; J22 += dNs[k] * lc[k][1]; }
    double det = J11 * J22 - J12 * J21;
    if (std::fabs(det) < 1e-12) return;
    double i11 = J22 / det, i12 = -J12 / det, i21 = -J21 / det, i22 = J11 / det;
    double rx = 0, sx = 0, ry = 0, sy = 0;
    for (int k = 0; k < 4; ++k) { rx += dNr[k] * Mc[k][0]; sx += dNs[k] * Mc[k][0]; ry += dNr[k] * Mc[k][1]; sy += dNs[k] * Mc[k][1]; }
    double eq[2] = {i11 * rx + i12 * sx, i21 * ry + i22 * sy};
    for (int i = 0; i < 2; ++i)
        if (std::isfinite(eq[i]) && std::fabs(eq[i]) < std::fabs(Q[i])) Q[i] = eq[i];
}

// quad4_is_axis_aligned_rectangle (FEMKernels.jl:5050-5077), tol 1e-8.
bool q4_is_rectangle(const double lc[4][2]) {
    const double tol = 1e-8;
    double e[4][2];
    for (int k = 0; k < 4; ++k) { int n = (k + 1) % 4; e[k][0] = lc[n][0] - lc[k][0]; e[k][1] = lc[n][1] - lc[k][1]; }
    double L[4], Lmax = 1e-12;
    for (int k = 0; k < 4; ++k) { L[k] = std::sqrt(e[k][0] * e[k][0] + e[k][1] * e[k][1]); Lmax = std::max(Lmax, L[k]); }
    double as = Lmax * Lmax;
    auto cr = [&](int a, int b) { return e[a][0] * e[b][1] - e[a][1] * e[b][0]; };
    auto dt = [&](int a, int b) { return e[a][0] * e[b][0] + e[a][1] * e[b][1]; };
    if (std::fabs(cr(0, 2)) > tol * as || std::fabs(cr(1, 3)) > tol * as) return false;
    if (std::fabs(dt(0, 1)) > tol * as || std::fabs(dt(1, 2)) > tol * as || std::fabs(dt(2, 3)) > tol * as ||
        std::fabs(dt(3, 0)) > tol * as)
        return false;
    if (std::fabs(L[0] - L[2]) > tol * Lmax || std::fabs(L[1] - L[3]) > tol * Lmax) return false;
    return true;
}

// CQUAD4 branch of recover_shell_stresses! (stress_recovery.jl:179-302).
void q4_recover(const double lc[4][2], const double u[24], double E, double nu, double h, double br, bool pressure_deck,
                ShellRec &R) {
    double eps[4][3], kap[4][3];
    if (!q4_stress_strain(lc, u, E, nu, h, br, R, eps, kap)) { R = ShellRec(); R.ok = false; return; }
    q4_corner_forces(E, nu, h, br, eps, kap, R.Nc, R.Mc);
    double Qo[2] = {R.Q[0], R.Q[1]};
    if (std::fabs(br) > 1e-12) q4_equilibrium_blend(lc, R.Mc, Qo);
    // _quad4_pressure_resultant_moment_scale (stress_recovery.jl:131-161)
    double scale = 1.0;
    if (pressure_deck && std::fabs(br) > 1e-12 && q4_is_rectangle(lc)) {
        double mq = std::max(std::fabs(Qo[0]), std::fabs(Qo[1]));
        double mn = std::max(std::fabs(R.N[0]), std::max(std::fabs(R.N[1]), std::fabs(R.N[2])));
        if (mq > 1e-8 && !(mn > std::max(1e-6, 1e-4 * mq))) scale = 0.99;
    }
    if (scale != 1.0)
        for (int c = 0; c < 3; ++c) {
            R.M[c] *= scale;
            for (int k = 0; k < 4; ++k) R.Mc[k][c] *= scale;
        }
    for (int k = 0; k < 4; ++k) R.Mc[k][2] = R.M[2];
    R.Q[0] = Qo[0];
    R.Q[1] = Qo[1];
}

// CTRIA3 macro recovery: tria3_plate_macro_data (FEMKernels.jl:7157-7209) with
// the recovery constitutive set of tria3_plate_macro_shear_resultant /
// tria3_plate_macro_average_moment (:7225-7305: Cm = D h, Cb = D h^3/12,
// Cs = 5/6 G h, G = E / 2(1 + nu), k6rot 100), then stress_strain_quad4 on each
// virtual quad with only its plate dofs.  Area-weighted sums of the quads'
// moments and shears; false where a factorisation raises.
bool t3_macro_fields(const double lc[3][2], const double u[18], double E, double nu, double h, double br, double Msum[3],
                     double Qsum[2], double &Asum) {
    double x[3] = {lc[0][0], lc[1][0], lc[2][0]}, y[3] = {lc[0][1], lc[1][1], lc[2][1]};
    double pts[7][2];
    for (int i = 0; i < 3; ++i) { pts[i][0] = x[i]; pts[i][1] = y[i]; }
    pts[3][0] = (x[0] + x[1]) / 2; pts[3][1] = (y[0] + y[1]) / 2;
    pts[4][0] = (x[1] + x[2]) / 2; pts[4][1] = (y[1] + y[2]) / 2;
    pts[5][0] = (x[2] + x[0]) / 2; pts[5][1] = (y[2] + y[0]) / 2;
    pts[6][0] = (x[0] + x[1] + x[2]) / 3; pts[6][1] = (y[0] + y[1] + y[2]) / 3;
    const int quads[3][4] = {{0, 3, 6, 5}, {1, 4, 6, 3}, {2, 5, 6, 4}};
    const int pd[12] = {2, 3, 4, 8, 9, 10, 14, 15, 16, 20, 21, 22};
    double D[3][3], Cm[3][3], Cb[3][3], Cs[2][2];
    plane_stress_D(E, nu, D);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Cm[i][j] = D[i][j] * h; Cb[i][j] = D[i][j] * (h * h * h / 12.0); }
    double G = E / (2.0 * (1.0 + nu));
    Cs[0][0] = Cs[1][1] = 5.0 / 6.0 * G * h;
    Cs[0][1] = Cs[1][0] = 0.0;
    double K21[21][21] = {};
    for (int q = 0; q < 3; ++q) {
        double qc[4][2];
        for (int k = 0; k < 4; ++k) { qc[k][0] = pts[quads[q][k]][0]; qc[k][1] = pts[quads[q][k]][1]; }
        double Kq[24][24];
        q4_stiffness(qc, Cm, Cb, Cs, h, G, 100.0, 1.0, /*bending_incomp=*/false, /*membrane_incomp=*/true, Kq);
        int ed[12];
        for (int k = 0; k < 4; ++k)
            for (int dd = 0; dd < 3; ++dd) ed[3 * k + dd] = 3 * quads[q][k] + dd;
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) K21[ed[i]][ed[j]] += Kq[pd[i]][pd[j]];
    }
    double Kii[144], Aint[12 * 9];
    for (int i = 0; i < 12; ++i) {
        for (int j = 0; j < 12; ++j) Kii[i * 12 + j] = K21[9 + i][9 + j];
        for (int j = 0; j < 9; ++j) Aint[i * 9 + j] = K21[9 + i][j];
    }
    if (!lu_solve(12, 9, Kii, Aint)) return false;
    const int up[9] = {2, 3, 4, 8, 9, 10, 14, 15, 16};
    double ua[21];
    for (int i = 0; i < 9; ++i) ua[i] = u[up[i]];
    for (int i = 0; i < 12; ++i) {
        double s = 0.0;
        for (int j = 0; j < 9; ++j) s += -Aint[i * 9 + j] * ua[j];
        ua[9 + i] = s;
    }
    Msum[0] = Msum[1] = Msum[2] = 0.0;
    Qsum[0] = Qsum[1] = 0.0;
    Asum = 0.0;
    for (int q = 0; q < 3; ++q) {
        double qc[4][2], uq[24] = {};
        for (int k = 0; k < 4; ++k) {
            qc[k][0] = pts[quads[q][k]][0]; qc[k][1] = pts[quads[q][k]][1];
            for (int dd = 0; dd < 3; ++dd) uq[pd[3 * k + dd]] = ua[3 * quads[q][k] + dd];
        }
        ShellRec Rq;
        double eps[4][3], kap[4][3];
        if (!q4_stress_strain(qc, uq, E, nu, h, br, Rq, eps, kap)) return false;
        // _tria3_virtual_quad_area (FEMKernels.jl:7151-7155)
        double a1 = (qc[1][0] - qc[0][0]) * (qc[3][1] - qc[0][1]) - (qc[3][0] - qc[0][0]) * (qc[1][1] - qc[0][1]);
        double a2 = (qc[2][0] - qc[1][0]) * (qc[3][1] - qc[1][1]) - (qc[3][0] - qc[1][0]) * (qc[2][1] - qc[1][1]);
        double area = (std::fabs(a1) + std::fabs(a2)) / 2;
        for (int c = 0; c < 3; ++c) Msum[c] += area * Rq.M[c];
        for (int c = 0; c < 2; ++c) Qsum[c] += area * Rq.Q[c];
        Asum += area;
    }
    return true;
}

// CTRIA3 branch of recover_shell_stresses! (stress_recovery.jl:303-354):
// stress_strain_tria3 (FEMKernels.jl:7391-7432) and, for macro weight w > 0,
// _blend_tria3_macro_bending_iso! (stress_recovery.jl:53-86).
void t3_recover(const double lc[3][2], const double u[18], double E, double nu, double h, double br, double w, ShellRec &R) {
    R = ShellRec();
    double x[3] = {lc[0][0], lc[1][0], lc[2][0]}, y[3] = {lc[0][1], lc[1][1], lc[2][1]};
    double A = 0.5 * std::fabs(x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]));
    if (A < 1e-12) return;  // the reference returns zeros for a degenerate triangle
    double b[3] = {(y[1] - y[2]) / (2 * A), (y[2] - y[0]) / (2 * A), (y[0] - y[1]) / (2 * A)};
    double c[3] = {(x[2] - x[1]) / (2 * A), (x[0] - x[2]) / (2 * A), (x[1] - x[0]) / (2 * A)};
    double eps[3] = {0, 0, 0}, kap[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        double ux = u[6 * i], uy = u[6 * i + 1], rx = u[6 * i + 3], ry = u[6 * i + 4];
        eps[0] += b[i] * ux; eps[1] += c[i] * uy; eps[2] += c[i] * ux + b[i] * uy;
        kap[0] += b[i] * ry; kap[1] += -c[i] * rx; kap[2] += c[i] * ry - b[i] * rx;
    }
    double D[3][3], De[3], Dk[3];
    plane_stress_D(E, nu, D);
    mv3(D, eps, De);
    mv3(D, kap, Dk);
    for (int k = 0; k < 3; ++k) { R.N[k] = De[k] * h; R.M[k] = -br * Dk[k] * (h * h * h / 12.0); }
    double Msum[3] = {0, 0, 0}, Qsum[2] = {0, 0}, Asum = 0.0;
    bool have_macro = false;
    if (br > 1e-12) {
        if (!t3_macro_fields(lc, u, E, nu, h, br, Msum, Qsum, Asum)) { R = ShellRec(); R.ok = false; return; }
        have_macro = true;
        if (Asum > 1e-12) { R.Q[0] = Qsum[0] / Asum; R.Q[1] = Qsum[1] / Asum; }
    }
    for (int k = 0; k < 3; ++k) { R.ez1[k] = eps[k] + (-h / 2.0) * kap[k]; R.ez2[k] = eps[k] + (h / 2.0) * kap[k]; }
    mv3(D, R.ez1, R.sz1);
    mv3(D, R.ez2, R.sz2);
    if (w > 0.0 && std::fabs(br) > 1e-12 && have_macro) {
        double Mm[3] = {0, 0, 0};
        if (Asum > 1e-12)
            for (int k = 0; k < 3; ++k) Mm[k] = Msum[k] / Asum;
        if (std::isfinite(Mm[0]) && std::isfinite(Mm[1]) && std::isfinite(Mm[2])) {
            double Mb[3], Dm[9], rhs[3];
            for (int k = 0; k < 3; ++k) Mb[k] = (1.0 - w) * R.M[k] + w * Mm[k];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Dm[3 * i + j] = D[i][j];
            for (int k = 0; k < 3; ++k) rhs[k] = Mb[k];
            lu_solve(3, 1, Dm, rhs);
            double kb[3], em[3];
            for (int k = 0; k < 3; ++k) {
                kb[k] = -(12.0 / (br * h * h * h)) * rhs[k];
                em[k] = (R.ez1[k] + R.ez2[k]) / 2.0;
            }
            for (int k = 0; k < 3; ++k) {
                R.M[k] = Mb[k];
                R.ez1[k] = em[k] + (-h / 2.0) * kb[k];
                R.ez2[k] = em[k] + (h / 2.0) * kb[k];
            }
            mv3(D, R.ez1, R.sz1);
            mv3(D, R.ez2, R.sz2);
        }
    }
}

// _tria3_shell_macro_blend_weights (stress_recovery.jl:20-51): edges counted
// over every CQUAD4 and CTRIA3; w = clamp((shared edges - 1) / 2, 0, 1).
void t3_macro_weights(const jfg_model_desc *d, std::vector<double> &w) {
    std::map<std::pair<int32_t, int32_t>, int> cnt;
    auto key = [](int32_t a, int32_t b) { return a < b ? std::make_pair(a, b) : std::make_pair(b, a); };
    for (int64_t e = 0; e < d->n_quad4; ++e)
        for (int k = 0; k < 4; ++k) cnt[key(d->quad4_nodes[4 * e + k], d->quad4_nodes[4 * e + (k + 1) % 4])] += 1;
    for (int64_t e = 0; e < d->n_tria3; ++e)
        for (int k = 0; k < 3; ++k) cnt[key(d->tria3_nodes[3 * e + k], d->tria3_nodes[3 * e + (k + 1) % 3])] += 1;
    w.assign(d->n_tria3, 0.0);
    for (int64_t e = 0; e < d->n_tria3; ++e) {
        int shared = 0;
        for (int k = 0; k < 3; ++k) shared += cnt[key(d->tria3_nodes[3 * e + k], d->tria3_nodes[3 * e + (k + 1) % 3])] > 1;
        w[e] = std::min(1.0, std::max(0.0, (shared - 1) / 2.0));
    }
}

void write_shell_rec(const ShellRec &R, double *o) {
    std::fill(o, o + JFG_SHELL_REC, 0.0);
    if (!R.ok) return;
    for (int k = 0; k < 3; ++k) {
        o[k] = R.N[k]; o[3 + k] = R.M[k]; o[8 + k] = R.sz1[k]; o[11 + k] = R.sz2[k]; o[14 + k] = R.ez1[k]; o[17 + k] = R.ez2[k];
    }
    o[6] = R.Q[0]; o[7] = R.Q[1];
    // compute_principal_2d (FEMKernels.jl:5921-5925), first root
    double s11 = R.sz1[0], s22 = R.sz1[1], s12 = R.sz1[2];
    o[20] = (s11 + s22) / 2.0 + std::sqrt(((s11 - s22) / 2.0) * ((s11 - s22) / 2.0) + s12 * s12);
    o[21] = 1.0;
    for (int k = 0; k < 4; ++k)
        for (int c = 0; c < 3; ++c) { o[22 + 3 * k + c] = R.Nc[k][c]; o[34 + 3 * k + c] = R.Mc[k][c]; }
    auto vm = [](const double *s) { return std::sqrt(s[0] * s[0] - s[0] * s[1] + s[1] * s[1] + 3 * s[2] * s[2]); };
    o[46] = vm(R.sz1);
    o[47] = vm(R.sz2);
}

// CBAR/CBEAM loop body of recover_bar_stresses! (stress_recovery.jl:446-503):
// forces_frame3d (FEMKernels.jl:215-229) on the offset-aware local
// displacements, axial stress and the section-point stresses.
void bar_recover(const jfg_model_desc *d, int64_t e, const double *u, const double *pts, double *o) {
    std::fill(o, o + JFG_BAR_REC, 0.0);
    double L, T12[12][12];
    bool off;
    if (!bar_setup(d, e, L, T12, off)) return;
    const int32_t *nd = d->bar_nodes + 2 * e;
    double ub[12] = {};
    for (int k = 0; k < 2; ++k) {
        const double *ug = u + 6 * (int64_t)nd[k];
        for (int dd = 0; dd < 6; ++dd)
            for (int q = 0; q < 6; ++q) ub[6 * k + dd] += T12[6 * k + dd][6 * k + q] * ug[q];
    }
    double A, Iy, Iz, I12, J, E, G, Asy, Asz;
    bar_section(d->bar_prop + JFG_BAR_PROP * e, A, Iy, Iz, I12, J, E, G, Asy, Asz);
    double k[12][12], f[12];
    frame3d_stiffness(L, A, Iy, Iz, J, E, G, Asy, Asz, I12, k);
    for (int i = 0; i < 12; ++i) {
        double s = 0.0;
        for (int q = 0; q < 12; ++q) s += k[i][q] * ub[q];
        f[i] = s;
    }
    o[0] = f[6]; o[1] = -f[1]; o[2] = -f[2]; o[3] = -f[3];
    o[4] = -f[5]; o[5] = f[4]; o[6] = f[11]; o[7] = -f[10];
    o[8] = std::fabs(A) > 1e-30 ? f[6] / A : 0.0;
    if (pts) {
        const double *p = pts + JFG_BAR_POINTS * e;
        double den = Iz * Iy - I12 * I12;
        for (int end = 0; end < 2; ++end) {
            double m1 = end == 0 ? o[4] : o[6], m2 = end == 0 ? o[5] : o[7];
            for (int j = 0; j < 4; ++j) {
                double yj = p[2 * j], zj = p[2 * j + 1];
                double s = std::fabs(den) > 1e-30 ? ((m1 * Iy - m2 * I12) * yj + (m2 * Iz - m1 * I12) * zj) / den
                                                  : m1 * yj / std::max(Iz, 1e-30) + m2 * zj / std::max(Iy, 1e-30);
                o[9 + 4 * end + j] = p[8] * s;
            }
        }
    }
    o[17] = 1.0;
}

// ---------------------------------------------------------------------------
// exported oracle API (test infrastructure)
// ---------------------------------------------------------------------------

struct OracleCSC {
    std::vector<int64_t> colptr, rowval;
    std::vector<double> nzval, orig_diag, abs_sums;
    double max_elem_stiff = 0.0;
    double t_elements = 0.0, t_sparse = 0.0;  // seconds: element loops; redistribution + sparse()
    std::string err;
};

bool g_abs_sums = false;  // also compute per-entry sums of |term| (tests only)

double now_s() {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}

// Element triplets of KG before constraints (assembly.jl:4382-6634), element
// order quads (576 each), trias (324 each), bars (144 each, zero-length bars
// dropped).  Returns nonzero where the reference raises.
int kg_element_triplets(const jfg_model_desc *d, const double *u, Triplets &t, std::string &err) {
    int st = check_predicates(d, err);
    if (st) return st;
    int64_t nq = d->n_quad4, nt = d->n_tria3, nb = d->n_bar;
    // CBAR/CBEAM with offsets: the reference's u_bar extraction indexes
    // T12[6+dd, 9+d] for d = 4..6, which is out of bounds for the 12x12 T12
    // and raises a BoundsError (assembly.jl:6322-6327, :6398-6403).
    for (int64_t e = 0; e < nb; ++e) {
        double L, T12[12][12];
        bool off;
        if (bar_setup(d, e, L, T12, off) && off) {
            err = "assemble_geometric_stiffness raises BoundsError for CBAR/CBEAM with offsets (assembly.jl:6326)";
            return JFG_ERR_REFERENCE_RAISES;
        }
    }
    size_t total = (size_t)nq * 576 + (size_t)nt * 324 + (size_t)nb * 144;
    t.I.resize(total); t.J.resize(total); t.V.resize(total);
    if (g_abs_sums) t.M.assign(total, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nq; ++e) {
        const int32_t *nd = d->quad4_nodes + 4 * e;
        const double *p[4];
        for (int k = 0; k < 4; ++k) p[k] = d->coords + 3 * nd[k];
        double v1[3], v2[3], v3[3];
        q4_frame(p[0], p[1], p[2], p[3], v1, v2, v3);
        double c[3];
        for (int i = 0; i < 3; ++i) c[i] = (p[0][i] + p[1][i] + p[2][i] + p[3][i]) / 4.0;
        double lc[4][2];
        for (int k = 0; k < 4; ++k) {
            double dd[3];
            sub3(p[k], c, dd);
            lc[k][0] = dot3(dd, v1); lc[k][1] = dot3(dd, v2);
        }
        double Q[36];
        node_blocks(d, nd, 4, v1, v2, v3, Q);
        // u_elem = T u_global (assembly.jl:5176-5185)
        double ue[24];
        for (int k = 0; k < 4; ++k) {
            const double *ug = u + 6 * (int64_t)nd[k];
            for (int dd = 0; dd < 3; ++dd) {
                ue[6 * k + dd] = Q[9 * k + 3 * dd] * ug[0] + Q[9 * k + 3 * dd + 1] * ug[1] + Q[9 * k + 3 * dd + 2] * ug[2];
                ue[6 * k + 3 + dd] = Q[9 * k + 3 * dd] * ug[3] + Q[9 * k + 3 * dd + 1] * ug[4] + Q[9 * k + 3 * dd + 2] * ug[5];
            }
        }
        const double *pr = d->quad4_prop + JFG_SHELL_PROP * e;
        double h = pr[0], E = pr[1], nu = pr[2];
        double cm = E / (1 - nu * nu);
        double Cm[3][3] = {{cm * 1.0 * h, cm * nu * h, 0.0}, {cm * nu * h, cm * 1.0 * h, 0.0}, {0.0, 0.0, cm * ((1 - nu) / 2) * h}};
        double Ngp[4][3], sig[4][3];
        q4_membrane_force_field(lc, ue, Cm, Ngp);
        for (int g = 0; g < 4; ++g)
            for (int cc = 0; cc < 3; ++cc) sig[g][cc] = Ngp[g][cc] / h;
        double Kl[24][24], G[576];
        q4_geometric_stiffness(lc, sig, h, Cm, Kl);
        transform_sym(4, Q, &Kl[0][0], G);
        for (int k = 0; k < 4; ++k) {
            int dd = 6 * k + 5;
            for (int r = 0; r < 24; ++r) { G[r * 24 + dd] = 0.0; G[dd * 24 + r] = 0.0; }
        }
        size_t base = (size_t)e * 576;
        if (g_abs_sums) {
            double us[24], Ml[24][24], Mg[576];
            local_u_scale(4, nd, Q, u, us);
            q4_kg_scale(lc, us, Cm, h, sig, Ml);
            transform_sym_abs(4, Q, &Ml[0][0], Mg);
            int q = 0;
            for (int cc = 0; cc < 24; ++cc)
                for (int rr = 0; rr < 24; ++rr, ++q) t.M[base + q] = (rr % 6 == 5 || cc % 6 == 5) ? 0.0 : Mg[rr * 24 + cc];
        }
        int cnt = 0;
        for (int cc = 0; cc < 24; ++cc)
            for (int rr = 0; rr < 24; ++rr) {
                t.I[base + cnt] = 6 * (int64_t)nd[rr / 6] + rr % 6;
                t.J[base + cnt] = 6 * (int64_t)nd[cc / 6] + cc % 6;
                t.V[base + cnt] = G[rr * 24 + cc];
                ++cnt;
            }
    }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nt; ++e) {
        const int32_t *nd = d->tria3_nodes + 3 * e;
        const double *p1 = d->coords + 3 * nd[0], *p2 = d->coords + 3 * nd[1], *p3 = d->coords + 3 * nd[2];
        double v1[3], v2[3], v3[3];
        t3_frame(p1, p2, p3, v1, v2, v3);
        double c[3];
        for (int i = 0; i < 3; ++i) c[i] = (p1[i] + p2[i] + p3[i]) / 3.0;
        const double *ps[3] = {p1, p2, p3};
        double lc[3][2];
        for (int k = 0; k < 3; ++k) {
            double dd[3];
            sub3(ps[k], c, dd);
            lc[k][0] = dot3(dd, v1); lc[k][1] = dot3(dd, v2);
        }
        double Q[27];
        node_blocks(d, nd, 3, v1, v2, v3, Q);
        double ue[18];
        for (int k = 0; k < 3; ++k) {
            const double *ug = u + 6 * (int64_t)nd[k];
            for (int dd = 0; dd < 3; ++dd) {
                ue[6 * k + dd] = Q[9 * k + 3 * dd] * ug[0] + Q[9 * k + 3 * dd + 1] * ug[1] + Q[9 * k + 3 * dd + 2] * ug[2];
                ue[6 * k + 3 + dd] = Q[9 * k + 3 * dd] * ug[3] + Q[9 * k + 3 * dd + 1] * ug[4] + Q[9 * k + 3 * dd + 2] * ug[5];
            }
        }
        const double *pr = d->tria3_prop + JFG_SHELL_PROP * e;
        double h = pr[0], E = pr[1], nu = pr[2];
        double Kl[18][18] = {};
        double x[3] = {lc[0][0], lc[1][0], lc[2][0]}, y[3] = {lc[0][1], lc[1][1], lc[2][1]};
        double A = 0.5 * std::fabs(x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]));
        if (A >= 1e-12 && h >= 1e-30) {
            // stress_strain_tria3 membrane part (FEMKernels.jl:7391-7404)
            double b[3] = {(y[1] - y[2]) / (2 * A), (y[2] - y[0]) / (2 * A), (y[0] - y[1]) / (2 * A)};
            double cv[3] = {(x[2] - x[1]) / (2 * A), (x[0] - x[2]) / (2 * A), (x[1] - x[0]) / (2 * A)};
            double um[6] = {ue[0], ue[1], ue[6], ue[7], ue[12], ue[13]};
            double eps[3] = {0, 0, 0};
            for (int i = 0; i < 3; ++i) {
                eps[0] += b[i] * um[2 * i];
                eps[1] += cv[i] * um[2 * i + 1];
                eps[2] += cv[i] * um[2 * i] + b[i] * um[2 * i + 1];
            }
            double cm = E / (1 - nu * nu);
            double D[3][3] = {{cm, cm * nu, 0.0}, {cm * nu, cm, 0.0}, {0.0, 0.0, cm * (1 - nu) / 2}};
            double N[3];
            for (int i = 0; i < 3; ++i) N[i] = (D[i][0] * eps[0] + D[i][1] * eps[1] + D[i][2] * eps[2]) * h;
            double sxx = N[0] / h, syy = N[1] / h, sxy = N[2] / h;
            // geometric_stiffness_tria3, non-curvature branch (FEMKernels.jl:8083-8097)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double val = h * A * (sxx * b[i] * b[j] + syy * cv[i] * cv[j] + sxy * (b[i] * cv[j] + cv[i] * b[j]));
                    for (int dd = 0; dd < 3; ++dd) Kl[6 * i + dd][6 * j + dd] += val;
                }
            if (g_abs_sums) {
                // rounding scale: the CST stress over the magnitudes of its strain terms
                double us[18], em[3] = {0, 0, 0}, Ml[18][18] = {}, Mg[324];
                local_u_scale(3, nd, Q, u, us);
                for (int i = 0; i < 3; ++i) {
                    em[0] += std::fabs(b[i]) * us[6 * i];
                    em[1] += std::fabs(cv[i]) * us[6 * i + 1];
                    em[2] += std::fabs(cv[i]) * us[6 * i] + std::fabs(b[i]) * us[6 * i + 1];
                }
                double sm[3];
                for (int r = 0; r < 3; ++r) sm[r] = std::fabs(D[r][0]) * em[0] + std::fabs(D[r][1]) * em[1] + std::fabs(D[r][2]) * em[2];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        const double mv = h * A * (sm[0] * std::fabs(b[i] * b[j]) + sm[1] * std::fabs(cv[i] * cv[j]) +
                                                   sm[2] * (std::fabs(b[i] * cv[j]) + std::fabs(cv[i] * b[j])));
                        for (int dd = 0; dd < 3; ++dd) Ml[6 * i + dd][6 * j + dd] = mv;
                    }
                transform_sym_abs(3, Q, &Ml[0][0], Mg);
                const size_t mb = (size_t)nq * 576 + (size_t)e * 324;
                int q = 0;
                for (int cc = 0; cc < 18; ++cc)
                    for (int rr = 0; rr < 18; ++rr, ++q) t.M[mb + q] = (rr % 6 == 5 || cc % 6 == 5) ? 0.0 : Mg[rr * 18 + cc];
            }
        }
        double G[324];
        transform_sym(3, Q, &Kl[0][0], G);
        for (int k = 0; k < 3; ++k) {
            int dd = 6 * k + 5;
            for (int r = 0; r < 18; ++r) { G[r * 18 + dd] = 0.0; G[dd * 18 + r] = 0.0; }
        }
        size_t base = (size_t)nq * 576 + (size_t)e * 324;
        int cnt = 0;
        for (int cc = 0; cc < 18; ++cc)
            for (int rr = 0; rr < 18; ++rr) {
                t.I[base + cnt] = 6 * (int64_t)nd[rr / 6] + rr % 6;
                t.J[base + cnt] = 6 * (int64_t)nd[cc / 6] + cc % 6;
                t.V[base + cnt] = G[rr * 18 + cc];
                ++cnt;
            }
    }
    std::vector<char> bar_ok(nb, 1);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nb; ++e) {
        double L, T12[12][12];
        bool off;
        if (!bar_setup(d, e, L, T12, off)) { bar_ok[e] = 0; continue; }
        const int32_t *nd = d->bar_nodes + 2 * e;
        double ub[12] = {};
        for (int k = 0; k < 2; ++k) {
            const double *ug = u + 6 * (int64_t)nd[k];
            for (int dd = 0; dd < 6; ++dd)
                for (int q = 0; q < 6; ++q) ub[6 * k + dd] += T12[6 * k + dd][6 * k + q] * ug[q];
        }
        double A, Iy, Iz, I12, J, E, G, Asy, Asz;
        bar_section(d->bar_prop + JFG_BAR_PROP * e, A, Iy, Iz, I12, J, E, G, Asy, Asz);
        double k[12][12];
        frame3d_stiffness(L, A, Iy, Iz, J, E, G, Asy, Asz, I12, k);
        double P = 0.0;
        for (int q = 0; q < 12; ++q) P += k[6][q] * ub[q];
        if (g_abs_sums) {
            // rounding scale of P: the sum k[6][q] ub[q] over the magnitudes
            // of its terms, each ub[q] itself a sum T u
            double Pm = 0.0;
            for (int q = 0; q < 12; ++q) {
                double um = 0.0;
                const int kq = q / 6;
                for (int l = 0; l < 6; ++l) um += std::fabs(T12[q][6 * kq + l] * u[6 * (int64_t)nd[kq] + l]);
                Pm += std::fabs(k[6][q]) * um;
            }
            double kg1[12][12], Mb[144];
            frame3d_geometric(L, 1.0, kg1);
            for (int i = 0; i < 12; ++i)
                for (int j = 0; j < 12; ++j) {
                    double s = 0.0;
                    for (int l = 0; l < 12; ++l)
                        for (int q = 0; q < 12; ++q) s += std::fabs(T12[l][i] * kg1[l][q] * T12[q][j]);
                    Mb[i * 12 + j] = Pm * s;
                }
            size_t base = (size_t)nq * 576 + (size_t)nt * 324 + (size_t)e * 144;
            int cnt = 0;
            for (int cc = 0; cc < 12; ++cc)
                for (int rr = 0; rr < 12; ++rr) t.M[base + cnt++] = Mb[rr * 12 + cc];
        }
        double kg[12][12], tmp[144], Kb[144];
        frame3d_geometric(L, P, kg);
        mul(tmp, &kg[0][0], &T12[0][0], 12, 12, 12);
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) {
                double s = 0.0;
                for (int l = 0; l < 12; ++l) s += T12[l][i] * tmp[l * 12 + j];
                Kb[i * 12 + j] = s;
            }
        size_t base = (size_t)nq * 576 + (size_t)nt * 324 + (size_t)e * 144;
        int cnt = 0;
        for (int cc = 0; cc < 12; ++cc)
            for (int rr = 0; rr < 12; ++rr) {
                t.I[base + cnt] = 6 * (int64_t)nd[rr / 6] + rr % 6;
                t.J[base + cnt] = 6 * (int64_t)nd[cc / 6] + cc % 6;
                t.V[base + cnt] = Kb[rr * 12 + cc];
                ++cnt;
            }
    }
    {
        size_t nbase = (size_t)nq * 576 + (size_t)nt * 324;
        if (g_abs_sums)  // a shell value with no stress term (A or h below the cutoffs) is 0; keep |V| there
            for (size_t q = 0; q < nbase; ++q) t.M[q] = std::max(t.M[q], std::fabs(t.V[q]));
        bool any = false;
        for (int64_t e = 0; e < nb; ++e) any |= !bar_ok[e];
        if (any) {
            Triplets u2;
            u2.I.assign(t.I.begin(), t.I.begin() + nbase); u2.J.assign(t.J.begin(), t.J.begin() + nbase); u2.V.assign(t.V.begin(), t.V.begin() + nbase);
            if (g_abs_sums) u2.M.assign(t.M.begin(), t.M.begin() + nbase);
            for (int64_t e = 0; e < nb; ++e)
                if (bar_ok[e])
                    for (int q = 0; q < 144; ++q) {
                        size_t s = nbase + e * 144 + q;
                        u2.I.push_back(t.I[s]); u2.J.push_back(t.J[s]); u2.V.push_back(t.V[s]);
                        if (g_abs_sums) u2.M.push_back(t.M[s]);
                    }
            t = std::move(u2);
        }
    }
    return 0;
}

extern "C" {

// Element-level entry points (local frame), used by tests on single elements.
void oracle_q4_stiffness_local(const double *lc8, const double *prop7, double k6rot, double *Ke576) {
    double lc[4][2], Cm[3][3], Cb[3][3], Cs[2][2];
    for (int k = 0; k < 4; ++k) { lc[k][0] = lc8[2 * k]; lc[k][1] = lc8[2 * k + 1]; }
    shell_constitutive(prop7, Cm, Cb, Cs);
    double br = prop7[4];
    double ek6 = br <= 1e-12 ? 0.0 : k6rot, eds = br <= 1e-12 ? 0.0 : 1.0;
    q4_stiffness(lc, Cm, Cb, Cs, prop7[0], prop7[1], ek6, eds, true, true, (double(*)[24])Ke576);
}

void oracle_t3_stiffness_local(const double *lc6, const double *prop7, double k6rot, double *Ke324) {
    double lc[3][2], Cm[3][3], Cb[3][3], Cs[2][2];
    for (int k = 0; k < 3; ++k) { lc[k][0] = lc6[2 * k]; lc[k][1] = lc6[2 * k + 1]; }
    shell_constitutive(prop7, Cm, Cb, Cs);
    double br = prop7[4];
    t3_stiffness(lc, Cm, Cb, Cs, prop7[0], prop7[6], br, br <= 1e-12 ? 0.0 : k6rot, (double(*)[18])Ke324);
}

// Element-level shell-thickness derivatives (local frame).
void oracle_q4_generic_local(const double *lc8, double E, double nu, double h, double *Ke576, double *dKe576) {
    double lc[4][2];
    for (int k = 0; k < 4; ++k) { lc[k][0] = lc8[2 * k]; lc[k][1] = lc8[2 * k + 1]; }
    q4_generic(lc, E, nu, h, (double(*)[24])Ke576, (double(*)[24])dKe576);
}
void oracle_t3_generic_local(const double *lc6, double E, double nu, double h, double *Ke324, double *dKe324) {
    double lc[3][2];
    for (int k = 0; k < 3; ++k) { lc[k][0] = lc6[2 * k]; lc[k][1] = lc6[2 * k + 1]; }
    if (Ke324) t3_generic(lc, E, nu, h, (double(*)[18])Ke324);
    if (dKe324) t3_generic_dkdh(lc, E, nu, h, (double(*)[18])dKe324);
}

// Shell-thickness sensitivities over a model (dKdx.jl:193-250), element
// thickness, E and nu from each element's property record:
//   c_q4[e] / c_t3[e] = a_e' T_e' dK_e/dh T_e b_e          (a, b: ndof)
//   load += T_e' dK_e/dh T_e u_e over elements with mask != 0 (load: ndof,
//   zeroed here; null masks select nothing).
// Any output or input pointer may be null to skip that part.
void oracle_dkdh(const jfg_model_desc *d, const double *a, const double *b, double *c_q4, double *c_t3, const double *u,
                 const uint8_t *mask_q4, const uint8_t *mask_t3, double *load) {
    const int64_t ndof = 6 * d->n_nodes;
    if (load) std::fill(load, load + ndof, 0.0);
    for (int type = 0; type < 2; ++type) {
        const int nn = type == 0 ? 4 : 3, nd6 = 6 * nn;
        const int64_t ne = type == 0 ? d->n_quad4 : d->n_tria3;
        const int32_t *nodes = type == 0 ? d->quad4_nodes : d->tria3_nodes;
        const double *prop = type == 0 ? d->quad4_prop : d->tria3_prop;
        double *cout = type == 0 ? c_q4 : c_t3;
        const uint8_t *mask = type == 0 ? mask_q4 : mask_t3;
        for (int64_t e = 0; e < ne; ++e) {
            const bool want_c = cout && a && b, want_f = load && u && mask && mask[e];
            if (!want_c && !want_f) continue;
            const int32_t *nd = nodes + nn * e;
            const double *pr = prop + JFG_SHELL_PROP * e;
            double lc[4][2], Q[36], dK[24 * 24];
            shell_setup(d, nd, nn, lc, Q);
            if (nn == 4) q4_generic(lc, pr[1], pr[2], pr[0], nullptr, (double(*)[24])dK);
            else {
                double lc3[3][2] = {{lc[0][0], lc[0][1]}, {lc[1][0], lc[1][1]}, {lc[2][0], lc[2][1]}};
                t3_generic_dkdh(lc3, pr[1], pr[2], pr[0], (double(*)[18])dK);
            }
            if (want_c) {
                double al[24], bl[24], s = 0.0;
                to_local(nn, Q, a, nd, al);
                to_local(nn, Q, b, nd, bl);
                for (int i = 0; i < nd6; ++i) {
                    double t = 0.0;
                    for (int c = 0; c < nd6; ++c) t += dK[nd6 * i + c] * bl[c];
                    s += al[i] * t;
                }
                cout[e] = s;
            }
            if (want_f) {
                double ul[24], fl[24];
                to_local(nn, Q, u, nd, ul);
                for (int i = 0; i < nd6; ++i) {
                    double t = 0.0;
                    for (int c = 0; c < nd6; ++c) t += dK[nd6 * i + c] * ul[c];
                    fl[i] = t;
                }
                // f_global = T' f_local, scattered to the element's dofs
                for (int k = 0; k < nn; ++k)
                    for (int half = 0; half < 2; ++half)
                        for (int c = 0; c < 3; ++c) {
                            double s = 0.0;
                            for (int r = 0; r < 3; ++r) s += Q[9 * k + 3 * r + c] * fl[6 * k + 3 * half + r];
                            load[6 * (int64_t)nd[k] + 3 * half + c] += s;
                        }
            }
        }
    }
}

// SOL 101 output recovery over a model (records as in jfem_gpu.h,
// JFG_SHELL_REC per shell -- CQUAD4s then CTRIA3s -- and JFG_BAR_REC per bar).
void oracle_recover(const jfg_model_desc *d, const double *u, const double *bar_points, int32_t flags,
                    double *shell_out, double *bar_out) {
    const bool pressure_deck = (flags & JFG_RECOVER_PRESSURE_DECK) && d->n_bar == 0 && d->n_rbe2 == 0;
    if (shell_out) {
        std::vector<double> w;
        t3_macro_weights(d, w);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < d->n_quad4 + d->n_tria3; ++i) {
            const bool quad = i < d->n_quad4;
            const int64_t e = quad ? i : i - d->n_quad4;
            const int nn = quad ? 4 : 3;
            const int32_t *nd = (quad ? d->quad4_nodes : d->tria3_nodes) + nn * e;
            const double *pr = (quad ? d->quad4_prop : d->tria3_prop) + JFG_SHELL_PROP * e;
            double lc[4][2], Q[36], ul[24];
            shell_setup(d, nd, nn, lc, Q);
            to_local(nn, Q, u, nd, ul);
            ShellRec R;
            if (quad) q4_recover(lc, ul, pr[1], pr[2], pr[0], pr[4], pressure_deck, R);
            else {
                double lc3[3][2] = {{lc[0][0], lc[0][1]}, {lc[1][0], lc[1][1]}, {lc[2][0], lc[2][1]}};
                t3_recover(lc3, ul, pr[1], pr[2], pr[0], pr[4], w[e], R);
            }
            write_shell_rec(R, shell_out + JFG_SHELL_REC * i);
        }
    }
    if (bar_out)
        for (int64_t e = 0; e < d->n_bar; ++e) bar_recover(d, e, u, bar_points, bar_out + JFG_BAR_REC * e);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Element triplets of K (before constraints), element order: quads, trias, bars.
// Returns 0 or a jfg status; *handle receives an OracleCSC.
int oracle_assemble_k(const jfg_model_desc *d, void **handle) {
    auto *out = new OracleCSC();
    *handle = out;
    int st = check_predicates(d, out->err);
    if (st) return st;
    const double t0 = now_s();
    int64_t nq = d->n_quad4, nt = d->n_tria3, nb = d->n_bar;
    Triplets t;
    size_t total = (size_t)nq * 576 + (size_t)nt * 324 + (size_t)nb * 144;
    t.I.resize(total); t.J.resize(total); t.V.resize(total);
    // CQUAD4 loop (assembly.jl:2657-3852)
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nq; ++e) {
        const int32_t *nd = d->quad4_nodes + 4 * e;
        const double *p[4];
        for (int k = 0; k < 4; ++k) p[k] = d->coords + 3 * nd[k];
        double v1[3], v2[3], v3[3];
        q4_frame(p[0], p[1], p[2], p[3], v1, v2, v3);
        double c[3];
        for (int i = 0; i < 3; ++i) c[i] = (p[0][i] + p[1][i] + p[2][i] + p[3][i]) / 4.0;
        double lc[4][2];
        for (int k = 0; k < 4; ++k) {
            double dd[3];
            sub3(p[k], c, dd);
            lc[k][0] = dot3(dd, v1); lc[k][1] = dot3(dd, v2);
        }
        const double *pr = d->quad4_prop + JFG_SHELL_PROP * e;
        double Cm[3][3], Cb[3][3], Cs[2][2];
        shell_constitutive(pr, Cm, Cb, Cs);
        double br = pr[4];
        double k6 = br <= 1e-12 ? 0.0 : d->k6rot, ds = br <= 1e-12 ? 0.0 : 1.0;
        double Ke[24][24];
        // elem_membrane_incomp is true for flat isotropic shells (assembly.jl:3393)
        q4_stiffness(lc, Cm, Cb, Cs, pr[0], pr[1], k6, ds, true, true, Ke);
        double Q[36], G[576];
        node_blocks(d, nd, 4, v1, v2, v3, Q);
        transform_sym(4, Q, &Ke[0][0], G);
        size_t base = (size_t)e * 576;
        int cnt = 0;
        for (int cc = 0; cc < 24; ++cc)
            for (int rr = 0; rr < 24; ++rr) {
                t.I[base + cnt] = 6 * (int64_t)nd[rr / 6] + rr % 6;
                t.J[base + cnt] = 6 * (int64_t)nd[cc / 6] + cc % 6;
                t.V[base + cnt] = G[rr * 24 + cc];
                ++cnt;
            }
    }
    // CTRIA3 loop (assembly.jl:3866-3955)
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nt; ++e) {
        const int32_t *nd = d->tria3_nodes + 3 * e;
        const double *p1 = d->coords + 3 * nd[0], *p2 = d->coords + 3 * nd[1], *p3 = d->coords + 3 * nd[2];
        double v1[3], v2[3], v3[3];
        t3_frame(p1, p2, p3, v1, v2, v3);
        double c[3];
        for (int i = 0; i < 3; ++i) c[i] = (p1[i] + p2[i] + p3[i]) / 3.0;
        const double *ps[3] = {p1, p2, p3};
        double lc[3][2];
        for (int k = 0; k < 3; ++k) {
            double dd[3];
            sub3(ps[k], c, dd);
            lc[k][0] = dot3(dd, v1); lc[k][1] = dot3(dd, v2);
        }
        const double *pr = d->tria3_prop + JFG_SHELL_PROP * e;
        double Cm[3][3], Cb[3][3], Cs[2][2];
        shell_constitutive(pr, Cm, Cb, Cs);
        double br = pr[4];
        double Ke[18][18];
        t3_stiffness(lc, Cm, Cb, Cs, pr[0], pr[6], br, br <= 1e-12 ? 0.0 : d->k6rot, Ke);
        double Q[27], G[324];
        node_blocks(d, nd, 3, v1, v2, v3, Q);
        transform_sym(3, Q, &Ke[0][0], G);
        size_t base = (size_t)nq * 576 + (size_t)e * 324;
        int cnt = 0;
        for (int cc = 0; cc < 18; ++cc)
            for (int rr = 0; rr < 18; ++rr) {
                t.I[base + cnt] = 6 * (int64_t)nd[rr / 6] + rr % 6;
                t.J[base + cnt] = 6 * (int64_t)nd[cc / 6] + cc % 6;
                t.V[base + cnt] = G[rr * 18 + cc];
                ++cnt;
            }
    }
    // CBAR / CBEAM (assembly.jl:3961-4092)
    std::vector<char> bar_ok(nb, 1);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nb; ++e) {
        double L, T12[12][12];
        bool off;
        size_t base = (size_t)nq * 576 + (size_t)nt * 324 + (size_t)e * 144;
        if (!bar_setup(d, e, L, T12, off)) { bar_ok[e] = 0; continue; }
        double A, Iy, Iz, I12, J, E, G, Asy, Asz;
        bar_section(d->bar_prop + JFG_BAR_PROP * e, A, Iy, Iz, I12, J, E, G, Asy, Asz);
        double k[12][12], tmp[144], Kg[144];
        frame3d_stiffness(L, A, Iy, Iz, J, E, G, Asy, Asz, I12, k);
        mul(tmp, &k[0][0], &T12[0][0], 12, 12, 12);
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) {
                double s = 0.0;
                for (int l = 0; l < 12; ++l) s += T12[l][i] * tmp[l * 12 + j];
                Kg[i * 12 + j] = s;
            }
        const int32_t *nd = d->bar_nodes + 2 * e;
        int cnt = 0;
        for (int cc = 0; cc < 12; ++cc)
            for (int rr = 0; rr < 12; ++rr) {
                t.I[base + cnt] = 6 * (int64_t)nd[rr / 6] + rr % 6;
                t.J[base + cnt] = 6 * (int64_t)nd[cc / 6] + cc % 6;
                t.V[base + cnt] = Kg[rr * 12 + cc];
                ++cnt;
            }
    }
    // zero-length bars are skipped (no triplets): compact
    {
        Triplets u;
        size_t nbase = (size_t)nq * 576 + (size_t)nt * 324;
        bool any = false;
        for (int64_t e = 0; e < nb; ++e) any |= !bar_ok[e];
        if (any) {
            u.I.assign(t.I.begin(), t.I.begin() + nbase); u.J.assign(t.J.begin(), t.J.begin() + nbase); u.V.assign(t.V.begin(), t.V.begin() + nbase);
            for (int64_t e = 0; e < nb; ++e)
                if (bar_ok[e])
                    for (int q = 0; q < 144; ++q) { size_t s = nbase + e * 144 + q; u.I.push_back(t.I[s]); u.J.push_back(t.J[s]); u.V.push_back(t.V[s]); }
            t = std::move(u);
        }
    }
    // max_elem_stiff and orig_diag before constraints (assembly.jl:4353-4364)
    double mx = 0.0;
    for (double v : t.V) mx = std::max(mx, std::fabs(v));
    out->max_elem_stiff = mx;
    out->orig_diag.assign(6 * d->n_nodes, 0.0);
    for (size_t k = 0; k < t.V.size(); ++k)
        if (t.I[k] == t.J[k]) out->orig_diag[t.I[k]] += t.V[k];
    const double t1 = now_s();
    constrain_and_csc(d, t, out->colptr, out->rowval, out->nzval, g_abs_sums ? &out->abs_sums : nullptr);
    out->t_elements = t1 - t0;
    out->t_sparse = now_s() - t1;
    return 0;
}

// KG assembly (assembly.jl:4382-6634), element order quads, trias, bars.
int oracle_assemble_kg(const jfg_model_desc *d, const double *u, void **handle) {
    auto *out = new OracleCSC();
    *handle = out;
    Triplets t;
    const double t0 = now_s();
    int st = kg_element_triplets(d, u, t, out->err);
    if (st) return st;
    const double t1 = now_s();
    constrain_and_csc(d, t, out->colptr, out->rowval, out->nzval, g_abs_sums ? &out->abs_sums : nullptr);
    out->t_elements = t1 - t0;
    out->t_sparse = now_s() - t1;
    return 0;
}

// Per-element contractions a_e' KG_e(u) b_e of every CQUAD4 and CTRIA3: the
// element matrices of the KG assembly before constraints.  With a = b = phi,
// c_e / h_e is the thickness sensitivity phi' dKG_e/dh phi of the reference's
// _dKg_dx_phi_thickness (adjoint_buckling.jl:2079-2150; KG is linear in h at
// fixed u).  Returns nonzero where the KG assembly raises.
int oracle_kg_contract(const jfg_model_desc *d, const double *u, const double *a, const double *b, double *c_q4,
                       double *c_t3) {
    Triplets t;
    std::string err;
    int st = kg_element_triplets(d, u, t, err);
    if (st) return st;
    for (int64_t e = 0; e < d->n_quad4; ++e) {
        double s = 0.0;
        for (size_t q = 576 * (size_t)e; q < 576 * (size_t)(e + 1); ++q) s += a[t.I[q]] * t.V[q] * b[t.J[q]];
        if (c_q4) c_q4[e] = s;
    }
    const size_t base = 576 * (size_t)d->n_quad4;
    for (int64_t e = 0; e < d->n_tria3; ++e) {
        double s = 0.0;
        for (size_t q = base + 324 * (size_t)e; q < base + 324 * (size_t)(e + 1); ++q) s += a[t.I[q]] * t.V[q] * b[t.J[q]];
        if (c_t3) c_t3[e] = s;
    }
    return 0;
}

int64_t oracle_nnz(void *h) { return (int64_t)((OracleCSC *)h)->nzval.size(); }
int64_t oracle_ndof(void *h) { return (int64_t)((OracleCSC *)h)->colptr.size() - 1; }
const char *oracle_error(void *h) { return ((OracleCSC *)h)->err.c_str(); }
double oracle_max_elem_stiff(void *h) { return ((OracleCSC *)h)->max_elem_stiff; }
void oracle_fetch(void *h, int64_t *colptr, int64_t *rowval, double *nzval, double *orig_diag) {
    auto *o = (OracleCSC *)h;
    if (colptr) std::memcpy(colptr, o->colptr.data(), sizeof(int64_t) * o->colptr.size());
    if (rowval) std::memcpy(rowval, o->rowval.data(), sizeof(int64_t) * o->rowval.size());
    if (nzval) std::memcpy(nzval, o->nzval.data(), sizeof(double) * o->nzval.size());
    if (orig_diag && !o->orig_diag.empty()) std::memcpy(orig_diag, o->orig_diag.data(), sizeof(double) * o->orig_diag.size());
}
void oracle_free(void *h) { delete (OracleCSC *)h; }
// Per-entry sums of |term| of the next assemblies (tests only; 0 = off).
void oracle_set_abs_sums(int on) { g_abs_sums = on != 0; }
int oracle_fetch_abs_sums(void *h, double *out) {
    auto *o = (OracleCSC *)h;
    if (o->abs_sums.size() != o->nzval.size()) return 1;
    std::memcpy(out, o->abs_sums.data(), sizeof(double) * o->abs_sums.size());
    return 0;
}
// Seconds spent in the element loops and in redistribution + sparse().
void oracle_phase_seconds(void *h, double *out2) {
    out2[0] = ((OracleCSC *)h)->t_elements;
    out2[1] = ((OracleCSC *)h)->t_sparse;
}

// rbe3_map as returned by assemble_stiffness (constraints.jl:319-322), 1-based
int64_t oracle_constraint_map(const jfg_model_desc *d, int64_t *dep, int64_t *ptr, int64_t *ind, double *coef) {
    auto mp = rbe2_map(d);
    int64_t n = 0, t = 0;
    if (ptr) ptr[0] = 0;
    for (auto &kv : mp) {
        if (dep) dep[n] = kv.first + 1;
        for (auto &p : kv.second) {
            if (ind) ind[t] = p.first + 1;
            if (coef) coef[t] = p.second;
            ++t;
        }
        ++n;
        if (ptr) ptr[n] = t;
    }
    return n;
}

}  // extern "C"
