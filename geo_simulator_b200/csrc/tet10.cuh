// Tet10 (10-node quadratic tetrahedron) device math.
//
// Local node order [v0 v1 v2 v3 e01 e12 e20 e03 e13 e23] (src/mesh/topology.rs:1-16,
// src/fem/basis.rs:5-13). Barycentric coordinates L0..L3 with L1, L2, L3 as the
// independent reference coordinates xi (basis.rs:196-223).
#pragma once

#include <cuda_runtime.h>

namespace geo {

// 4-point rule (quadrature.rs:24-38): L_q = b + (a - b) e_q, weight 1/24.
constexpr double kQa = 0.5854101966249685;
constexpr double kQb = 0.1381966011250105;
constexpr double kQw = 1.0 / 24.0;
// 5-point rule (quadrature.rs:44-59).
constexpr double kQ5a = 0.25, kQ5b = 1.0 / 6.0, kQ5c = 0.5;

// Edge k joins vertices kEdge[k][0] and kEdge[k][1] (topology.rs:41-50).
__host__ __device__ constexpr int edge_v(int k, int s) {
    return (k == 0) ? (s ? 1 : 0)
         : (k == 1) ? (s ? 2 : 1)
         : (k == 2) ? (s ? 0 : 2)
         : (k == 3) ? (s ? 3 : 0)
         : (k == 4) ? (s ? 3 : 1)
                    : (s ? 3 : 2);
}

// Barycentric coordinates of 4-point quadrature point q.
template <class T>
__host__ __device__ __forceinline__ void qp4(int q, T (&L)[4]) {
#pragma unroll
    for (int m = 0; m < 4; ++m) L[m] = (m == q) ? T(kQa) : T(kQb);
}

template <class T>
__host__ __device__ __forceinline__ void qp5(int q, T (&L)[4]) {
    if (q == 0) {
#pragma unroll
        for (int m = 0; m < 4; ++m) L[m] = T(kQ5a);
    } else {
        // points 1..4 put 0.5 on coordinate 4-q (quadrature.rs:51-55)
#pragma unroll
        for (int m = 0; m < 4; ++m) L[m] = (m == 4 - q) ? T(kQ5c) : T(kQ5b);
    }
}

__host__ __device__ __forceinline__ double qw5(int q) { return q == 0 ? -2.0 / 15.0 : 3.0 / 40.0; }

// Shape functions N_i(L), basis.rs:56-73.
template <class T>
__host__ __device__ __forceinline__ void shape_n(const T (&L)[4], T (&N)[10]) {
#pragma unroll
    for (int m = 0; m < 4; ++m) N[m] = L[m] * (T(2) * L[m] - T(1));
#pragma unroll
    for (int k = 0; k < 6; ++k) N[4 + k] = T(4) * L[edge_v(k, 0)] * L[edge_v(k, 1)];
}

// Reference gradient g_i = dN_i/dxi (xi = L1, L2, L3; L0 eliminated), i.e.
// dN_i/dL_a - dN_i/dL_0 for a = 1..3 (basis.rs:85-110, :206-208).
template <class T>
__host__ __device__ __forceinline__ void ref_grad(int i, const T (&L)[4], T (&g)[3]) {
    // dN_i/dL_m
    T d[4] = {T(0), T(0), T(0), T(0)};
    if (i < 4) {
        d[i] = T(4) * L[i] - T(1);
    } else {
        const int m = edge_v(i - 4, 0), n = edge_v(i - 4, 1);
        d[m] = T(4) * L[n];
        d[n] = T(4) * L[m];
    }
    g[0] = d[1] - d[0];
    g[1] = d[2] - d[0];
    g[2] = d[3] - d[0];
}

// Isoparametric Jacobian J[r][c] = d x_r / d xi_c from the 10 node coordinates
// (basis.rs:196-223).
template <class T>
__host__ __device__ __forceinline__ void jacobian10(const T (&X)[10][3], const T (&L)[4], T (&J)[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) J[r][c] = T(0);
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        T g[3];
        ref_grad(i, L, g);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) J[r][c] += X[i][r] * g[c];
    }
}

template <class T>
__host__ __device__ __forceinline__ T det3(const T (&J)[3][3]) {
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

// Adjugate (J^{-1} = adj / det).
template <class T>
__host__ __device__ __forceinline__ void adj3(const T (&J)[3][3], T (&A)[3][3]) {
    A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
    A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
    A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
    A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
}

// Cartesian gradient grad N_i = J^{-T} g_i (basis.rs:265-272), given Jinv.
template <class T>
__host__ __device__ __forceinline__ void cart_grad(const T (&Ji)[3][3], const T (&g)[3], T (&out)[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) out[a] = Ji[0][a] * g[0] + Ji[1][a] * g[1] + Ji[2][a] * g[2];
}

// ----------------------------------------------------------------------------
// Matrix-free building blocks (no reference counterpart; the reference forms
// K_e explicitly). For a scalar nodal field T_i the reference gradient at the
// 4-point quadrature point q is
//     h_m(q) = dT/dL_m = 4 (M L_q)_m - T_m,     grad_xi T = (h_1-h_0, h_2-h_0, h_3-h_0)
// with the symmetric 4x4 nodal matrix M_mm = T_m, M_mn = T_edge(m,n). With
// L_q = b + (a-b) e_q: h_m(q) = (4b S_m - T_m) + 4(a-b) M_mq, S_m = sum_n M_mn.
// The transpose maps QP fluxes v_q (3-vectors) back to nodal values.
// ----------------------------------------------------------------------------
template <class T>
struct RefGradQ4 {
    T base[4];  // 4b S_m - T_m
    T M[4][4];
};

// edge local index of the pair (m, n), m != n
__host__ __device__ constexpr int edge_of(int m, int n) {
    return ((m == 0 && n == 1) || (m == 1 && n == 0)) ? 4
         : ((m == 1 && n == 2) || (m == 2 && n == 1)) ? 5
         : ((m == 2 && n == 0) || (m == 0 && n == 2)) ? 6
         : ((m == 0 && n == 3) || (m == 3 && n == 0)) ? 7
         : ((m == 1 && n == 3) || (m == 3 && n == 1)) ? 8
                                                      : 9;
}

// grad_xi of the field te[10] at the four 4-point QPs: gq[q][a].
template <class T>
__device__ __forceinline__ void ref_grad_field_q4(const T (&te)[10], T (&gq)[4][3]) {
    const T B4 = T(4.0 * kQb), D4 = T(4.0 * (kQa - kQb));
    T M[4][4];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n) M[m][n] = (m == n) ? te[m] : te[edge_of(m, n)];
    T base[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) base[m] = B4 * (M[m][0] + M[m][1] + M[m][2] + M[m][3]) - te[m];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const T h0 = base[0] + D4 * M[0][q];
        gq[q][0] = base[1] + D4 * M[1][q] - h0;
        gq[q][1] = base[2] + D4 * M[2][q] - h0;
        gq[q][2] = base[3] + D4 * M[3][q] - h0;
    }
}

// Transpose of ref_grad_field_q4: y_i = sum_q g_i(L_q) . vq[q]  (writes y[10]).
template <class T>
__device__ __forceinline__ void ref_grad_transpose_q4(const T (&vq)[4][3], T (&y)[10]) {
    const T B4 = T(4.0 * kQb), D4 = T(4.0 * (kQa - kQb));
    T phi[4][4];  // phi[q][m]
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        phi[q][0] = -(vq[q][0] + vq[q][1] + vq[q][2]);
        phi[q][1] = vq[q][0];
        phi[q][2] = vq[q][1];
        phi[q][3] = vq[q][2];
    }
    T Phi[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) Phi[m] = phi[0][m] + phi[1][m] + phi[2][m] + phi[3][m];
#pragma unroll
    for (int m = 0; m < 4; ++m) y[m] = (B4 - T(1)) * Phi[m] + D4 * phi[m][m];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int m = edge_v(k, 0), n = edge_v(k, 1);
        y[4 + k] = B4 * (Phi[m] + Phi[n]) + D4 * (phi[n][m] + phi[m][n]);
    }
}

}  // namespace geo
