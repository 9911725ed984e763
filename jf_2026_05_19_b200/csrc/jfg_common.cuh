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
JFG_HD void normalize3(const double *a, double *o) {
    double n = sqrt(dot3(a, a));
    o[0] = a[0] / n; o[1] = a[1] / n; o[2] = a[2] / n;
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
JFG_HD void inv4_inplace(double A[16]) {
    double B[16];
    for (int i = 0; i < 16; ++i) B[i] = (i % 5 == 0) ? 1.0 : 0.0;
    for (int k = 0; k < 4; ++k) {
        int p = k;
        double best = fabs(A[4 * k + k]);
        for (int i = k + 1; i < 4; ++i) {
            double v = fabs(A[4 * i + k]);
            if (v > best) { best = v; p = i; }
        }
        if (p != k)
            for (int j = 0; j < 4; ++j) {
                double t = A[4 * k + j]; A[4 * k + j] = A[4 * p + j]; A[4 * p + j] = t;
                t = B[4 * k + j]; B[4 * k + j] = B[4 * p + j]; B[4 * p + j] = t;
            }
        double inv = 1.0 / A[4 * k + k];
        for (int j = 0; j < 4; ++j) { A[4 * k + j] *= inv; B[4 * k + j] *= inv; }
        for (int i = 0; i < 4; ++i) {
            if (i == k) continue;
            double f = A[4 * i + k];
            if (f != 0.0)
                for (int j = 0; j < 4; ++j) { A[4 * i + j] -= f * A[4 * k + j]; B[4 * i + j] -= f * B[4 * k + j]; }
        }
    }
    for (int i = 0; i < 16; ++i) A[i] = B[i];
}

// Order-independent max of non-negative doubles through their bit patterns.
JFG_D void atomic_max_nonneg(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

}  // namespace jfg
