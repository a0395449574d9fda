// Matrix-free Tet10 element kernels shared by the operator, the persistent PCG
// and the adjoint. No reference counterpart: the reference forms K_e
// explicitly (element.rs:23-61, mechanics/element.rs:33-65); these apply the
// same K_e to a vector without forming it.
#pragma once

#include "tet10.cuh"

namespace geo {

// Per-element geometric data ("qdata"), stored patch-major: for patch p, value j
// of the patch's element e sits at [(p * NQD + j) * kPatchElems + e]. Thermal: the symmetric 3x3 G = (k w / |det J|) adj(J) adj(J)^T packed
// as [xx xy xz yy yz zz], once for affine elements (NQ = 1) or per quadrature
// point (NQ = 4, curved elements). Elasticity: J^{-1} (9, row-major) and
// s = w |det J| E_e, once or per quadrature point.
template <class T, int NQ>
struct ThermalK {
    static constexpr int DPN = 1;
    static constexpr int NQD = 6 * NQ;

    // qd points at the element's first qdata value; value j sits at qd[j * stride]
    __device__ __forceinline__ static void apply(const T* __restrict__ qd, int64_t stride, T, T,
                                                 const T (&x)[10], T (&y)[10]) {
        // h_m(q) = base_m + D4 M_mq (M: nodal matrix), grad_xi = (h1-h0, h2-h0, h3-h0);
        // flux v_q = G grad_xi; phi_q = (-sum v, v); Phi = sum_q phi_q; then
        //   y_m = (B4 - 1) Phi_m + D4 phi_{m,m},  y_(mn) = B4 (Phi_m + Phi_n) + D4 (phi_{n,m} + phi_{m,n}).
        const T B4 = T(4.0 * kQb), D4 = T(4.0 * (kQa - kQb)), B4m1 = T(4.0 * kQb - 1.0);
        T base[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            T s = x[m];
#pragma unroll
            for (int n = 0; n < 4; ++n)
                if (n != m) s += x[edge_of(m, n)];
            base[m] = B4 * s - x[m];
        }
        T G[6];
        if (NQ == 1) {
#pragma unroll
            for (int j = 0; j < 6; ++j) G[j] = qd[j * stride];
        }
        T phi[4][4], Phi[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (NQ == 4) {
#pragma unroll
                for (int j = 0; j < 6; ++j) G[j] = qd[(6 * q + j) * stride];
            }
            T h[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) h[m] = base[m] + D4 * (m == q ? x[m] : x[edge_of(m, q)]);
            const T g0 = h[1] - h[0], g1 = h[2] - h[0], g2 = h[3] - h[0];
            const T v0 = G[0] * g0 + G[1] * g1 + G[2] * g2;
            const T v1 = G[1] * g0 + G[3] * g1 + G[4] * g2;
            const T v2 = G[2] * g0 + G[4] * g1 + G[5] * g2;
            phi[q][0] = -(v0 + v1 + v2);
            phi[q][1] = v0;
            phi[q][2] = v1;
            phi[q][3] = v2;
#pragma unroll
            for (int m = 0; m < 4; ++m) Phi[m] = q == 0 ? phi[0][m] : Phi[m] + phi[q][m];
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) y[m] = B4m1 * Phi[m] + D4 * phi[m][m];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int m = edge_v(k, 0), n = edge_v(k, 1);
            y[4 + k] = B4 * (Phi[m] + Phi[n]) + D4 * (phi[n][m] + phi[m][n]);
        }
    }
};

template <class T, int NQ>
struct ElasticK {
    static constexpr int DPN = 3;
    static constexpr int NQD = 10 * NQ;

    // x, y interleaved [3*i + c]; cl = nu/((1+nu)(1-2nu)), cm = 1/(2(1+nu))
    __device__ __forceinline__ static void apply(const T* __restrict__ qd, int64_t stride, T cl, T cm,
                                                 const T (&x)[30], T (&y)[30]) {
        const T B4 = T(4.0 * kQb), D4 = T(4.0 * (kQa - kQb)), B4m1 = T(4.0 * kQb - 1.0);
        T base[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                T s = x[3 * m + c];
#pragma unroll
                for (int n = 0; n < 4; ++n)
                    if (n != m) s += x[3 * edge_of(m, n) + c];
                base[c][m] = B4 * s - x[3 * m + c];
            }
#pragma unroll
        for (int i = 0; i < 30; ++i) y[i] = T(0);
        T Ji[9], s = T(0);
        if (NQ == 1) {
#pragma unroll
            for (int j = 0; j < 9; ++j) Ji[j] = qd[j * stride];
            s = qd[9 * stride];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (NQ == 4) {
#pragma unroll
                for (int j = 0; j < 9; ++j) Ji[j] = qd[(10 * q + j) * stride];
                s = qd[(10 * q + 9) * stride];
            }
            // displacement gradient F[c][b] = sum_a H[c][a] Ji[a][b]
            T F[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T h[4];
#pragma unroll
                for (int m = 0; m < 4; ++m)
                    h[m] = base[c][m] + D4 * (m == q ? x[3 * m + c] : x[3 * edge_of(m, q) + c]);
                const T H0 = h[1] - h[0], H1 = h[2] - h[0], H2 = h[3] - h[0];
#pragma unroll
                for (int b = 0; b < 3; ++b) F[c][b] = H0 * Ji[b] + H1 * Ji[3 + b] + H2 * Ji[6 + b];
            }
            const T tr = cl * (F[0][0] + F[1][1] + F[2][2]);
            T S[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int b = 0; b < 3; ++b) S[c][b] = s * (cm * (F[c][b] + F[b][c]) + (c == b ? tr : T(0)));
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                // P[c][a] = sum_b S[c][b] Ji[a][b]
                const T P0 = S[c][0] * Ji[0] + S[c][1] * Ji[1] + S[c][2] * Ji[2];
                const T P1 = S[c][0] * Ji[3] + S[c][1] * Ji[4] + S[c][2] * Ji[5];
                const T P2 = S[c][0] * Ji[6] + S[c][1] * Ji[7] + S[c][2] * Ji[8];
                const T phi[4] = {-(P0 + P1 + P2), P0, P1, P2};
#pragma unroll
                for (int m = 0; m < 4; ++m) y[3 * m + c] += (m == q ? B4m1 + D4 : B4m1) * phi[m];
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const int m = edge_v(k, 0), n = edge_v(k, 1);
                    T t = B4 * (phi[m] + phi[n]);
                    if (q == n) t += D4 * phi[m];
                    if (q == m) t += D4 * phi[n];
                    y[3 * (4 + k) + c] += t;
                }
            }
        }
    }
};

}  // namespace geo
