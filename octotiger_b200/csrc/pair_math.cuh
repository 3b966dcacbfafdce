// Per-pair arithmetic of the FMM cell-interaction kernels (device side).
//
// Two FP64 forms of the same interaction:
//   * Exact*: the operation sequence of the reference templates
//     (octotiger/multipole_interactions/kernel/compute_kernel_templates.hpp:67-391,
//      octotiger/monopole_interactions/kernel/monopole_kernel_templates.hpp:16-239)
//     with every product and sum an explicitly rounded IEEE operation
//     (__dmul_rn / __dadd_rn / __dsub_rn, IEEE division and square root), so
//     the result is bit-for-bit the reference's;
//   * Fast*: the same interaction with fused multiply-adds, the multinomial
//     factors folded into the partner moments at staging time (Scaled
//     moments: M[4..9] * factor/2, M[10..19] * factor/6), and the derivative
//     tensor built from one reciprocal square root.
// Moment order: M, Mx, My, Mz, Mxx, Mxy, Mxz, Myy, Myz, Mzz, Mxxx, Mxxy, Mxxz,
// Mxyy, Mxyz, Mxzz, Myyy, Myyz, Myzz, Mzzz (src/taylor.cpp:10-56).
#pragma once

#include <cuda_runtime.h>

namespace otfmm {

// Fused multiply-add with the precision of its operands (no promotion).
__device__ __forceinline__ float fmat(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmat(double a, double b, double c) { return __fma_rn(a, b, c); }

// factor[] of compute_kernel_templates.hpp:37-39 (multinomial multiplicities).
__host__ __device__ constexpr double factor_of(int k) {
    return (k == 5 || k == 6 || k == 8) ? 2.0
         : (k == 11 || k == 12 || k == 13 || k == 15 || k == 17 || k == 18) ? 3.0
         : (k == 14) ? 6.0 : 1.0;
}
// Octupole index reached from quadrupole 4+q along axis a.
__host__ __device__ constexpr int quad_axis(int q, int a) {
    return q == 0 ? 10 + a
         : q == 1 ? (a == 0 ? 11 : a == 1 ? 13 : 14)
         : q == 2 ? (a == 0 ? 12 : a == 1 ? 14 : 15)
         : q == 3 ? (a == 0 ? 13 : a == 1 ? 16 : 17)
         : q == 4 ? (a == 0 ? 14 : a == 1 ? 17 : 18)
                  : (a == 0 ? 15 : a == 1 ? 18 : 19);
}
// Quadrupole index of axes (a, b).
__host__ __device__ constexpr int quad_row(int a, int b) {
    return a == 0 ? 4 + b : a == 1 ? (b == 0 ? 5 : b == 1 ? 7 : 8) : (b == 0 ? 6 : b == 1 ? 8 : 9);
}
// D_upper operand of the angular correction for octupole 10+o and output j.
__host__ __device__ constexpr int upper_idx(int o, int j) {
    return o == 0 ? j
         : o == 1 ? (j == 0 ? 1 : j == 1 ? 3 : 4)
         : o == 2 ? (j == 0 ? 2 : j == 1 ? 4 : 5)
         : o == 3 ? (j == 0 ? 3 : j == 1 ? 6 : 7)
         : o == 4 ? (j == 0 ? 4 : j == 1 ? 7 : 8)
         : o == 5 ? (j == 0 ? 5 : j == 1 ? 8 : 9)
         : o == 6 ? (j == 0 ? 6 : j == 1 ? 10 : 11)
         : o == 7 ? (j == 0 ? 7 : j == 1 ? 11 : 12)
         : o == 8 ? (j == 0 ? 8 : j == 1 ? 12 : 13)
                  : (j == 0 ? 9 : j == 1 ? 13 : 14);
}

// ------------------------------------------------------------------ exact FP64
#define OT_MUL __dmul_rn
#define OT_ADD __dadd_rn
#define OT_SUB __dsub_rn

struct ExactDerivs {
    double d2, d3, X00, X11, X22;
    double D[20];
};

// compute_d_factors (:67-139)
__device__ __forceinline__ void exact_d_factors(const double dX[3], ExactDerivs& f) {
    f.X00 = OT_MUL(dX[0], dX[0]);
    f.X11 = OT_MUL(dX[1], dX[1]);
    f.X22 = OT_MUL(dX[2], dX[2]);
    const double r2 = OT_ADD(OT_ADD(f.X00, f.X11), f.X22);
    const double r2inv = __ddiv_rn(1.0, fmax(r2, 1.0e-20));
    const double d0 = -__dsqrt_rn(r2inv);
    const double d1 = OT_MUL(-d0, r2inv);
    const double d2 = OT_MUL(OT_MUL(-3.0, d1), r2inv);
    const double d3 = OT_MUL(OT_MUL(-5.0, d2), r2inv);
    f.d2 = d2;
    f.d3 = d3;
    double* D = f.D;
    D[0] = d0;
#pragma unroll
    for (int a = 0; a < 3; ++a) D[1 + a] = OT_MUL(dX[a], d1);
    const double X12 = OT_MUL(dX[1], dX[2]), X01 = OT_MUL(dX[0], dX[1]), X02 = OT_MUL(dX[0], dX[2]);
    D[4] = OT_ADD(OT_MUL(d2, f.X00), d1);
    D[5] = OT_MUL(d2, X01);
    D[6] = OT_MUL(d2, X02);
    D[7] = OT_ADD(OT_MUL(d2, f.X11), d1);
    D[8] = OT_MUL(d2, X12);
    D[9] = OT_ADD(OT_MUL(d2, f.X22), d1);
    const double d2x0 = OT_MUL(d2, dX[0]), d2x1 = OT_MUL(d2, dX[1]), d2x2 = OT_MUL(d2, dX[2]);
    D[10] = OT_ADD(OT_MUL(OT_MUL(d3, f.X00), dX[0]), OT_MUL(3.0, d2x0));
    D[11] = OT_ADD(OT_MUL(OT_MUL(d3, f.X00), dX[1]), d2x1);
    D[12] = OT_ADD(OT_MUL(OT_MUL(d3, f.X00), dX[2]), d2x2);
    D[13] = OT_ADD(OT_MUL(OT_MUL(d3, dX[0]), f.X11), d2x0);
    D[14] = OT_MUL(OT_MUL(d3, dX[0]), X12);
    D[15] = OT_ADD(OT_MUL(OT_MUL(d3, dX[0]), f.X22), d2x0);
    D[16] = OT_ADD(OT_MUL(OT_MUL(d3, f.X11), dX[1]), OT_MUL(3.0, d2x1));
    D[17] = OT_ADD(OT_MUL(OT_MUL(d3, f.X11), dX[2]), d2x2);
    D[18] = OT_ADD(OT_MUL(OT_MUL(d3, dX[1]), f.X22), d2x1);
    D[19] = OT_ADD(OT_MUL(OT_MUL(d3, f.X22), dX[2]), OT_MUL(3.0, d2x2));
}

// Fourth-order slice of the angular correction (:232-325).
__device__ __forceinline__ void exact_d_upper(const ExactDerivs& f, const double dX[3], double U[15]) {
    const double d2 = f.d2, d3 = f.d3;
    const double d3x00 = OT_MUL(d3, f.X00), d3x11 = OT_MUL(d3, f.X11), d3x22 = OT_MUL(d3, f.X22);
    const double d3x01 = OT_MUL(OT_MUL(d3, dX[0]), dX[1]);
    const double d3x02 = OT_MUL(OT_MUL(d3, dX[0]), dX[2]);
    const double d3x12 = OT_MUL(OT_MUL(d3, dX[1]), dX[2]);
    const double two_d2 = OT_MUL(2.0, d2);
    U[0] = OT_ADD(OT_ADD(OT_ADD(OT_MUL(OT_MUL(dX[0], dX[0]), d3), two_d2), d2), OT_MUL(5.0, d3x00));
    U[1] = OT_MUL(3.0, d3x01);
    U[2] = OT_MUL(3.0, d3x02);
    U[3] = OT_ADD(OT_ADD(d2, d3x11), d3x00);
    U[4] = d3x12;
    U[5] = OT_ADD(OT_ADD(d2, d3x22), d3x00);
    U[6] = OT_MUL(3.0, d3x01);
    U[7] = d3x02;
    U[8] = d3x01;
    U[9] = OT_MUL(3.0, d3x02);
    U[10] = OT_ADD(OT_ADD(OT_ADD(OT_MUL(OT_MUL(dX[1], dX[1]), d3), two_d2), d2), OT_MUL(5.0, d3x11));
    U[11] = OT_MUL(3.0, d3x12);
    U[12] = OT_ADD(OT_ADD(d2, d3x22), d3x11);
    U[13] = OT_MUL(3.0, d3x12);
    U[14] = OT_ADD(OT_ADD(OT_ADD(OT_MUL(OT_MUL(dX[2], dX[2]), d3), two_d2), d2), OT_MUL(5.0, d3x22));
}

__device__ __forceinline__ void exact_monopole_terms(const double* m, const double* D, double* L) {
#pragma unroll
    for (int a = 0; a < 4; ++a) L[a] = OT_ADD(L[a], OT_MUL(m[0], D[a]));
}
__device__ __forceinline__ void exact_dipole_terms(const double* m, const double* D, double* L) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        L[0] = OT_SUB(L[0], OT_MUL(m[1 + a], D[1 + a]));
#pragma unroll
        for (int b = 0; b < 3; ++b) L[1 + a] = OT_SUB(L[1 + a], OT_MUL(m[1 + a], D[quad_row(a, b)]));
    }
}
__device__ __forceinline__ void exact_quad_oct_terms(const double* m, const double* D, double* L) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int k = 4 + q;
        const double fh = factor_of(k) / 2.0;
        L[0] = OT_ADD(L[0], OT_MUL(m[k], OT_MUL(D[k], fh)));
#pragma unroll
        for (int a = 0; a < 3; ++a) L[1 + a] = OT_ADD(L[1 + a], OT_MUL(m[k], OT_MUL(D[quad_axis(q, a)], fh)));
    }
#pragma unroll
    for (int k = 10; k < 20; ++k) L[0] = OT_SUB(L[0], OT_MUL(m[k], OT_MUL(D[k], factor_of(k) / 6.0)));
}
__device__ __forceinline__ void exact_higher_terms(const double* m, const double* D, double* L) {
#pragma unroll
    for (int q = 0; q < 6; ++q) L[4 + q] = OT_ADD(L[4 + q], OT_MUL(m[0], D[4 + q]));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int q = 0; q < 6; ++q) L[4 + q] = OT_SUB(L[4 + q], OT_MUL(m[1 + a], D[quad_axis(q, a)]));
#pragma unroll
    for (int o = 0; o < 10; ++o) L[10 + o] = OT_ADD(L[10 + o], OT_MUL(m[0], D[10 + o]));
}

// compute_kernel_rho / compute_kernel_non_rho
template <bool RHO>
__device__ __forceinline__ void exact_m2l_pair(const double X[3], const double Y[3], const double mp[20],
                                               const double mc[20], double L[20], double Lc[3]) {
    const double dX[3] = {OT_SUB(X[0], Y[0]), OT_SUB(X[1], Y[1]), OT_SUB(X[2], Y[2])};
    ExactDerivs f;
    exact_d_factors(dX, f);
    exact_monopole_terms(mp, f.D, L);
    if (!RHO) exact_dipole_terms(mp, f.D, L);
    exact_quad_oct_terms(mp, f.D, L);
    exact_higher_terms(mp, f.D, L);
    if (RHO) {
        double U[15];
        exact_d_upper(f, dX, U);
        const double n0 = __ddiv_rn(mp[0], mc[0]);
#pragma unroll
        for (int o = 0; o < 10; ++o) {
            const double n0t = OT_SUB(mp[10 + o], OT_MUL(mc[10 + o], n0));
            const double f6 = factor_of(10 + o) / 6.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) Lc[j] = OT_SUB(Lc[j], OT_MUL(n0t, OT_MUL(U[upper_idx(o, j)], f6)));
        }
    }
}

// compute_kernel_p2m_rho / compute_kernel_p2m_non_rho
template <bool RHO>
__device__ __forceinline__ void exact_p2m_pair(const double X[3], const double Y[3], const double mp[20],
                                               double L[4], double Lc[3]) {
    const double dX[3] = {OT_SUB(X[0], Y[0]), OT_SUB(X[1], Y[1]), OT_SUB(X[2], Y[2])};
    ExactDerivs f;
    exact_d_factors(dX, f);
    exact_monopole_terms(mp, f.D, L);
    if (!RHO) exact_dipole_terms(mp, f.D, L);
    exact_quad_oct_terms(mp, f.D, L);
    if (RHO) {
        double U[15];
        exact_d_upper(f, dX, U);
#pragma unroll
        for (int o = 0; o < 10; ++o) {
            const double f6 = factor_of(10 + o) / 6.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) Lc[j] = OT_SUB(Lc[j], OT_MUL(mp[10 + o], OT_MUL(U[upper_idx(o, j)], f6)));
        }
    }
}

// ------------------------------------------------------------------ fast FP64
// Partner and cell moments are Scaled: m[4..9] *= factor/2, m[10..19] *= factor/6.
struct FastDerivs {
    double d2, d3, X00, X11, X22, X01, X02, X12;
    double D[20];
};

__device__ __forceinline__ void fast_d_factors(const double dX[3], FastDerivs& f) {
    f.X00 = dX[0] * dX[0];
    f.X11 = dX[1] * dX[1];
    f.X22 = dX[2] * dX[2];
    f.X01 = dX[0] * dX[1];
    f.X02 = dX[0] * dX[2];
    f.X12 = dX[1] * dX[2];
    const double r2 = fmax(f.X00 + f.X11 + f.X22, 1.0e-20);
    const double rs = rsqrt(r2);          // 1/r
    const double r2inv = rs * rs;
    const double d1 = rs * r2inv;         // -d0 * r2inv with d0 = -1/r
    const double d2 = -3.0 * d1 * r2inv;
    const double d3 = -5.0 * d2 * r2inv;
    f.d2 = d2;
    f.d3 = d3;
    double* D = f.D;
    D[0] = -rs;
    D[1] = dX[0] * d1;
    D[2] = dX[1] * d1;
    D[3] = dX[2] * d1;
    D[4] = fma(d2, f.X00, d1);
    D[5] = d2 * f.X01;
    D[6] = d2 * f.X02;
    D[7] = fma(d2, f.X11, d1);
    D[8] = d2 * f.X12;
    D[9] = fma(d2, f.X22, d1);
    const double d2_3 = 3.0 * d2;
    const double a0 = fma(d3, f.X00, d2), a1 = fma(d3, f.X11, d2), a2 = fma(d3, f.X22, d2);
    const double b0 = fma(d3, f.X00, d2_3), b1 = fma(d3, f.X11, d2_3), b2 = fma(d3, f.X22, d2_3);
    D[10] = dX[0] * b0;
    D[11] = dX[1] * a0;
    D[12] = dX[2] * a0;
    D[13] = dX[0] * a1;
    D[14] = d3 * dX[0] * f.X12;
    D[15] = dX[0] * a2;
    D[16] = dX[1] * b1;
    D[17] = dX[2] * a1;
    D[18] = dX[1] * a2;
    D[19] = dX[2] * b2;
}

// Derivative tensor of 1/r from dX and d0..d3 (any scalar type).
template <class T>
__device__ __forceinline__ void d_tensor(const T dX[3], T d0, T d1, T d2, T d3, T D[20]) {
    const T X00 = dX[0] * dX[0], X11 = dX[1] * dX[1], X22 = dX[2] * dX[2];
    const T X01 = dX[0] * dX[1], X02 = dX[0] * dX[2], X12 = dX[1] * dX[2];
    D[0] = d0;
    D[1] = dX[0] * d1;
    D[2] = dX[1] * d1;
    D[3] = dX[2] * d1;
    D[4] = fmat(d2, X00, d1);
    D[5] = d2 * X01;
    D[6] = d2 * X02;
    D[7] = fmat(d2, X11, d1);
    D[8] = d2 * X12;
    D[9] = fmat(d2, X22, d1);
    const T d2_3 = T(3) * d2;
    const T a0 = fmat(d3, X00, d2), a1 = fmat(d3, X11, d2), a2 = fmat(d3, X22, d2);
    const T b0 = fmat(d3, X00, d2_3), b1 = fmat(d3, X11, d2_3), b2 = fmat(d3, X22, d2_3);
    D[10] = dX[0] * b0;
    D[11] = dX[1] * a0;
    D[12] = dX[2] * a0;
    D[13] = dX[0] * a1;
    D[14] = d3 * dX[0] * X12;
    D[15] = dX[0] * a2;
    D[16] = dX[1] * b1;
    D[17] = dX[2] * a1;
    D[18] = dX[1] * a2;
    D[19] = dX[2] * b2;
}

// Contraction shared by M2L and P2M for L0..L3 (quadrupole/octupole partner
// moments; Scaled moments carry the factors): one FMA per term, straight
// into the accumulators.
template <class T>
__device__ __forceinline__ void fast_low_terms(const T* m, const T* D, T* L, bool dipole) {
#pragma unroll
    for (int a = 0; a < 4; ++a) L[a] = fmat(m[0], D[a], L[a]);
    if (dipole) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            L[0] = fmat(-m[1 + a], D[1 + a], L[0]);
#pragma unroll
            for (int b = 0; b < 3; ++b) L[1 + a] = fmat(-m[1 + a], D[quad_row(a, b)], L[1 + a]);
        }
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        L[0] = fmat(m[4 + q], D[4 + q], L[0]);
#pragma unroll
        for (int a = 0; a < 3; ++a) L[1 + a] = fmat(m[4 + q], D[quad_axis(q, a)], L[1 + a]);
    }
#pragma unroll
    for (int k = 10; k < 20; ++k) L[0] = fmat(-m[k], D[k], L[0]);
}

template <class T>
__device__ __forceinline__ void fast_high_terms(const T* m, const T* D, T* L) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        T t = fmat(m[0], D[4 + q], L[4 + q]);
#pragma unroll
        for (int a = 0; a < 3; ++a) t = fmat(-m[1 + a], D[quad_axis(q, a)], t);
        L[4 + q] = t;
    }
#pragma unroll
    for (int o = 0; o < 10; ++o) L[10 + o] = fmat(m[0], D[10 + o], L[10 + o]);
}

// Angular correction with Scaled octupoles g_k = f6_k (M_p - M_c n0).
__device__ __forceinline__ void fast_upper_correction(const FastDerivs& f, const double g[10], double Lc[3]) {
    const double d2 = f.d2, d3 = f.d3;
    const double e01 = d3 * f.X01, e02 = d3 * f.X02, e12 = d3 * f.X12;
    const double d3_6 = 6.0 * d3, d2_3 = 3.0 * d2;
    double U[15];
    U[0] = fma(d3_6, f.X00, d2_3);
    U[1] = 3.0 * e01;
    U[2] = 3.0 * e02;
    U[3] = fma(d3, f.X00 + f.X11, d2);
    U[4] = e12;
    U[5] = fma(d3, f.X00 + f.X22, d2);
    U[6] = U[1];
    U[7] = e02;
    U[8] = e01;
    U[9] = U[2];
    U[10] = fma(d3_6, f.X11, d2_3);
    U[11] = 3.0 * e12;
    U[12] = fma(d3, f.X11 + f.X22, d2);
    U[13] = U[11];
    U[14] = fma(d3_6, f.X22, d2_3);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        double t = Lc[j];
#pragma unroll
        for (int o = 0; o < 10; ++o) t = fma(-g[o], U[upper_idx(o, j)], t);
        Lc[j] = t;
    }
}

// mc holds the target cell's Scaled octupoles mc[10..19] and inv_m0 = 1/M_c.
template <bool RHO>
__device__ __forceinline__ void fast_m2l_pair(const double X[3], const double Y[3], const double mp[20],
                                              const double mc_oct[10], double inv_m0, double L[20], double Lc[3]) {
    const double dX[3] = {X[0] - Y[0], X[1] - Y[1], X[2] - Y[2]};
    FastDerivs f;
    fast_d_factors(dX, f);
    fast_low_terms(mp, f.D, L, !RHO);
    fast_high_terms(mp, f.D, L);
    if (RHO) {
        const double n0 = mp[0] * inv_m0;
        double g[10];
#pragma unroll
        for (int o = 0; o < 10; ++o) g[o] = fma(-mc_oct[o], n0, mp[10 + o]);
        fast_upper_correction(f, g, Lc);
    }
}

// Partner with mass only (monopole-only stencil entries, leaf neighbours).
template <bool RHO>
__device__ __forceinline__ void fast_m2l_mass_pair(const double X[3], const double Y[3], double m0,
                                                   const double mc_oct[10], double inv_m0, double L[20],
                                                   double Lc[3]) {
    const double dX[3] = {X[0] - Y[0], X[1] - Y[1], X[2] - Y[2]};
    FastDerivs f;
    fast_d_factors(dX, f);
#pragma unroll
    for (int a = 0; a < 20; ++a) L[a] = fma(m0, f.D[a], L[a]);
    if (RHO) {
        const double n0 = m0 * inv_m0;
        double g[10];
#pragma unroll
        for (int o = 0; o < 10; ++o) g[o] = -mc_oct[o] * n0;
        fast_upper_correction(f, g, Lc);
    }
}

// ------------------------------------------------------------------ FP32 split
// Inputs in units of the subgrid cell size dx (exact for dx = 2^-k): X, Y
// centres of mass / dx (FP64), partner moments M'_k = M_k dx^-n(k) with the
// factors folded in, FP32 copies mpf and FP64 octupoles mp_oct for L_c.
// The derivative factors d0..d3 and the angular correction stay FP64; the
// derivative tensor and the D.M contraction run in FP32 into accf.
template <bool RHO>
__device__ __forceinline__ void split_m2l_pair(const double X[3], const double Y[3], const float mpf[20], double m0,
                                               const double mp_oct[10], const double mc_oct[10], double inv_m0,
                                               float accf[20], double Lc[3]) {
    FastDerivs f;
    const double dX[3] = {X[0] - Y[0], X[1] - Y[1], X[2] - Y[2]};
    f.X00 = dX[0] * dX[0];
    f.X11 = dX[1] * dX[1];
    f.X22 = dX[2] * dX[2];
    f.X01 = dX[0] * dX[1];
    f.X02 = dX[0] * dX[2];
    f.X12 = dX[1] * dX[2];
    const double r2 = fmax(f.X00 + f.X11 + f.X22, 1.0e-20);
    // 1/r: FP32 hardware estimate refined by one FP64 Newton step
    // (relative error ~1e-14, far below what L_c needs)
    const float r2f = (float)r2;
    const float y0 = rsqrtf(r2f);
    const double y = (double)y0;
    const double rs = y * fma(-0.5 * r2 * y, y, 1.5);
    const double r2inv = rs * rs;
    const double d1 = rs * r2inv;
    f.d2 = -3.0 * d1 * r2inv;
    f.d3 = -5.0 * f.d2 * r2inv;
    // FP32 factors from the refined 1/r (one conversion)
    const float rsf = (float)rs;
    const float r2invf = rsf * rsf;
    const float d1f = rsf * r2invf;
    const float d2f = -3.0f * d1f * r2invf;
    const float d3f = -5.0f * d2f * r2invf;
    const float dXf[3] = {(float)dX[0], (float)dX[1], (float)dX[2]};
    float Df[20];
    d_tensor<float>(dXf, -rsf, d1f, d2f, d3f, Df);
    fast_low_terms<float>(mpf, Df, accf, !RHO);
    fast_high_terms<float>(mpf, Df, accf);
    if (RHO) {
        const double n0 = m0 * inv_m0;
        double g[10];
#pragma unroll
        for (int o = 0; o < 10; ++o) g[o] = fma(-mc_oct[o], n0, mp_oct[o]);
        fast_upper_correction(f, g, Lc);
    }
}

template <bool RHO>
__device__ __forceinline__ void fast_p2m_pair(const double X[3], const double Y[3], const double mp[20],
                                              double L[4], double Lc[3]) {
    const double dX[3] = {X[0] - Y[0], X[1] - Y[1], X[2] - Y[2]};
    FastDerivs f;
    fast_d_factors(dX, f);
    fast_low_terms(mp, f.D, L, !RHO);
    if (RHO) fast_upper_correction(f, mp + 10, Lc);
}

}   // namespace otfmm
