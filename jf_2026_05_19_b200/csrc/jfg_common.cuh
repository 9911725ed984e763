// jfg_common.cuh -- shared device helpers for the element kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define JFG_HD __host__ __device__ __forceinline__
#define JFG_D __device__ __forceinline__

namespace jfg {

// Packed upper-triangle index of (i, j), i <= j, in an n x n symmetric block.
JFG_HD int packed_index(int i, int j, int n) { return i * n - (i * (i - 1)) / 2 + (j - i); }
JFG_HD int packed_size(int n) { return n * (n + 1) / 2; }

JFG_HD void sub3(const double *a, const double *b, double *o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }
JFG_HD double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
JFG_HD void cross3(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
// a / |a| with one reciprocal square root (within an ulp or two of three
// divisions by sqrt(a.a)).
JFG_HD void normalize3(const double *a, double *o) {
#ifdef __CUDA_ARCH__
    const double r = rsqrt(dot3(a, a));
#else
    const double r = 1.0 / sqrt(dot3(a, a));
#endif
    o[0] = a[0] * r; o[1] = a[1] * r; o[2] = a[2] * r;
}

// Flatness predicate of the default CQUAD4 branch (assembly.jl:2824-2840):
// the largest distance of a corner from the mean plane through the centroid
// (normal d13 x d24) is below 1e-6 of the longer diagonal.  Host code
// (model build) and device code (the allocation-free entry point) share it.
JFG_HD bool q4_is_flat(const double *p1, const double *p2, const double *p3, const double *p4) {
    double d13[3], d24[3], n[3];
    sub3(p3, p1, d13);
    sub3(p4, p2, d24);
    cross3(d13, d24, n);
    const double len = sqrt(dot3(n, n));
    double maxdev = 0.0;
    if (len > 1e-12) {
        const double g[3] = {n[0] / len, n[1] / len, n[2] / len};
        const double *ps[4] = {p1, p2, p3, p4};
        for (int k = 0; k < 4; ++k) {
            double d[3];
            for (int i = 0; i < 3; ++i) d[i] = ps[k][i] - (p1[i] + p2[i] + p3[i] + p4[i]) / 4.0;
            maxdev = fmax(maxdev, fabs(dot3(d, g)));
        }
    }
    const double L = fmax(sqrt(dot3(d13, d13)), sqrt(dot3(d24, d24)));
    return maxdev < 1e-6 * fmax(L, 1e-12);
}

// CQUAD4 element frame in the reference's default ":diag" mode
// (shell_element_frame_quad4 / _with_normal, helpers.jl:1134-1193).
JFG_HD void q4_frame(const double *p1, const double *p2, const double *p3, const double *p4,
                     double v1[3], double v2[3], double v3[3]) {
    double gxi[3], geta[3], v3r[3];
    for (int i = 0; i < 3; ++i) {
        gxi[i] = 0.25 * (-p1[i] + p2[i] + p3[i] - p4[i]);
        geta[i] = 0.25 * (-p1[i] - p2[i] + p3[i] + p4[i]);
    }
    cross3(gxi, geta, v3r);
    double d13[3], d24[3];
    sub3(p3, p1, d13);
    sub3(p4, p2, d24);
    if (dot3(v3r, v3r) <= 1e-24) cross3(d13, d24, v3r);
    normalize3(v3r, v3);
    double d13n[3], d24n[3], xr[3];
    normalize3(d13, d13n);
    normalize3(d24, d24n);
    for (int i = 0; i < 3; ++i) xr[i] = d13n[i] - d24n[i];
    if (dot3(xr, xr) < 1e-20)
        for (int i = 0; i < 3; ++i) xr[i] = d13n[i] + d24n[i];
    double xp[3];
    double dv = dot3(xr, v3);
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

// CTRIA3 frame (shell_element_frame_fast, n == 3, helpers.jl:1195-1204).
JFG_HD void t3_frame(const double *p1, const double *p2, const double *p3, double v1[3], double v2[3], double v3[3]) {
    double e[3], f[3], c[3];
    sub3(p2, p1, e);
    normalize3(e, v1);
    sub3(p3, p1, f);
    cross3(v1, f, c);
    normalize3(c, v3);
    cross3(v3, v1, v2);
}

// Q = Rel * node_R (3x3, row-major), Rel rows = v1, v2, v3; R == nullptr means identity.
JFG_HD void node_block(const double v1[3], const double v2[3], const double v3[3], const double *R, double Q[9]) {
    const double *rows[3] = {v1, v2, v3};
    if (!R) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Q[3 * r + c] = rows[r][c];
        return;
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Q[3 * r + c] = rows[r][0] * R[c] + rows[r][1] * R[3 + c] + rows[r][2] * R[6 + c];
}

// In-place Gauss-Jordan inverse of a 4x4 (row-major) with partial pivoting.
// Fully unrolled with predicated row swaps, so both working matrices stay in
// registers.
JFG_HD void inv4_inplace(double A[16]) {
    double a[16], b[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) { a[i] = A[i]; b[i] = (i % 5 == 0) ? 1.0 : 0.0; }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int p = k;
        double best = fabs(a[5 * k]);
#pragma unroll
        for (int i = k + 1; i < 4; ++i) {
            double v = fabs(a[4 * i + k]);
            if (v > best) { best = v; p = i; }
        }
#pragma unroll
        for (int i = k + 1; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool sw = (p == i);
                double ta = a[4 * k + j], tb = b[4 * k + j];
                a[4 * k + j] = sw ? a[4 * i + j] : ta; a[4 * i + j] = sw ? ta : a[4 * i + j];
                b[4 * k + j] = sw ? b[4 * i + j] : tb; b[4 * i + j] = sw ? tb : b[4 * i + j];
            }
        const double inv = 1.0 / a[5 * k];
#pragma unroll
        for (int j = 0; j < 4; ++j) { a[4 * k + j] *= inv; b[4 * k + j] *= inv; }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (i == k) continue;
            const double f = a[4 * i + k];
#pragma unroll
            for (int j = 0; j < 4; ++j) { a[4 * i + j] -= f * a[4 * k + j]; b[4 * i + j] -= f * b[4 * k + j]; }
        }
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) A[i] = b[i];
}

// MacNeal residual-bending-flexibility compliance of one (virtual) quad for
// an isotropic shear matrix Cs = cs I (add_quad4_macneal_shear_rbf!,
// FEMKernels.jl:4715-4978).  With Cs off-diagonal zero, VGV is diagonal, so
// Z = sym(inv(sym(VGV)) + Zb) is block diagonal with 2x2 blocks on the
// xi-sampling rows (0, 1) and the eta-sampling rows (2, 3); neither block
// pivots (|z01| < z00 since 1/VGV > 0), so the reference's LU solve Z \ D
// reduces to two 2x2 eliminations whose factors are kept here.
struct MacNealZ {
    double z01, r00, f01, r11;  // rows 0-1: off-diagonal, 1/z00, z01/z00, 1/(z11 - f01 z01)
    double z23, r22, f23, r33;  // rows 2-3
};

// lq: corner local coordinates (4 x 2); Jp: |det J| at the four strain
// sampling points; cs: transverse shear stiffness; cb00, cb11: bending
// stiffness diagonal.
JFG_HD MacNealZ macneal_z(const double lq[4][2], const double Jp[4], double cs, double cb00, double cb11) {
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
    double flex_x = 1.0 / fmax(fabs(cb00), 1e-30), flex_y = 1.0 / fmax(fabs(cb11), 1e-30);
    double inv12A = 1.0 / (12.0 * A_elem);
    const double zb = 0.65;
    double zxu = zb * inv12A * Dx2 * flex_x, zxd = zb * inv12A * ap * Dx2 * flex_x;
    double zyu = zb * inv12A * Dy2 * flex_y, zyd = zb * inv12A * bp * Dy2 * flex_y;
    double vd[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double s = sqrt(2.0 * Jp[i]);
        double v = s * s * cs;
        vd[i] = v < 1e-30 ? 1e-30 : v;
    }
    MacNealZ z;
    double z00 = 1.0 / vd[0] + (zxu + zxd), z11 = 1.0 / vd[1] + (zxu + zxd);
    double z22 = 1.0 / vd[2] + (zyu + zyd), z33 = 1.0 / vd[3] + (zyu + zyd);
    z.z01 = zxu - zxd;
    z.r00 = 1.0 / z00;
    z.f01 = z.z01 / z00;
    z.r11 = 1.0 / (z11 - z.f01 * z.z01);
    z.z23 = zyu - zyd;
    z.r22 = 1.0 / z22;
    z.f23 = z.z23 / z22;
    z.r33 = 1.0 / (z33 - z.f23 * z.z23);
    return z;
}

// One column of Y = Z \ D from the matching column d of the sampling rows.
JFG_HD void macneal_y(const MacNealZ &z, const double d[4], double y[4]) {
    y[1] = (d[1] - z.f01 * d[0]) * z.r11;
    y[0] = (d[0] - z.z01 * y[1]) * z.r00;
    y[3] = (d[3] - z.f23 * d[2]) * z.r33;
    y[2] = (d[2] - z.z23 * y[3]) * z.r22;
}

// Order-independent max of non-negative doubles through their bit patterns.
JFG_D void atomic_max_nonneg(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

// Staged slots leave shared memory as bulk asynchronous copies (the copy
// engine moves a whole slot per instruction).  Both addresses are 16-byte
// aligned and the size a multiple of 16 bytes.  Each thread that wrote a
// slot's values runs slot_fence() before the copying thread, after a warp
// sync where those differ, issues slot_copy(); every copying thread runs
// slot_copies_read() before its shared memory is reused or released.
JFG_D void slot_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
JFG_D void slot_copy(double *dst, const double *src, uint32_t bytes) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(src));
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n\tcp.async.bulk.commit_group;"
                 :: "l"(dst), "r"(s), "r"(bytes) : "memory");
}
JFG_D void slot_copies_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// All but the most recent copy have read their shared memory (double-buffered staging).
JFG_D void slot_copies_read_but_last() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }

}  // namespace jfg
