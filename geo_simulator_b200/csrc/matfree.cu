// K5/K6/K7: matrix-free Tet10 operator, persistent Jacobi-PCG (FP64 and mixed
// FP32/FP64 with on-device residual refresh), and the adjoint element gradient.
//
// Operator: K_bc of apply_dirichlet_bcs (assembly.rs:168-230) applied to a
// vector without assembling K (assembly.rs:69-117 / :389-437):
//   free rows  y_i = sum_{j free} K_ij x_j,   Dirichlet rows y_i = char_diag x_i.
// Elements are processed patch by patch (see patches.h): a CTA gathers the
// patch's nodal values into shared memory, every thread applies K_e of its
// elements from the per-element qdata, accumulates into shared memory, and the
// patch flushes its nodes: plain stores for nodes no other patch touches,
// red.global.add for the shared ones (so the matrix-free result is not
// bit-reproducible in the last bit; the assembled path is).
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "matfree.cuh"
#include "patches.h"
#include "pcg_common.cuh"

struct geo_op;

namespace geo {

constexpr int kMfBS = 128;

enum ApplyMode : int { MODE_FREE = 0, MODE_LIFT = 1 };

struct PatchView {
    int64_t E, N;
    int n_patches, ucap, dpn;
    const int32_t* pe;
    const int32_t* po;
    const int32_t* pf;
    const int32_t* foreign;
    const uint16_t* lconn;
    const uint8_t* flags;
};

// One patch-ordered pass y (+)= K x over all patches handled by this block
// (patch = blockIdx.x, += gridDim.x). D-row outputs are left untouched; in
// MODE_FREE Dirichlet inputs are read as zero, in MODE_LIFT free inputs are.
// Returns this thread's share of x^T y over the elements (masked x).
template <class K, class T>
__device__ double element_phase(const PatchView& pv, const T* __restrict__ qd, T cl, T cm, const T* __restrict__ x,
                                T* __restrict__ y, void* smem_raw, int mode) {
    constexpr int DPN = K::DPN;
    T* sx = reinterpret_cast<T*>(smem_raw);
    T* sy = sx + pv.ucap * DPN;
    double dot = 0.0;
    for (int patch = blockIdx.x; patch < pv.n_patches; patch += gridDim.x) {
        const int e0 = pv.pe[patch], e1 = pv.pe[patch + 1];
        const int o0 = pv.po[patch], nown = pv.po[patch + 1] - o0;
        const int f0 = pv.pf[patch], nloc = nown + pv.pf[patch + 1] - f0;
        for (int u = threadIdx.x; u < nloc; u += blockDim.x) {
            const int node = u < nown ? o0 + u : pv.foreign[f0 + u - nown];
            const uint8_t fl = pv.flags[node];
#pragma unroll
            for (int c = 0; c < DPN; ++c) {
                T v = x[(int64_t)node * DPN + c];
                const bool dir = (fl >> c) & 1;
                if (mode == MODE_FREE ? dir : !dir) v = T(0);
                sx[u * DPN + c] = v;
                sy[u * DPN + c] = T(0);
            }
        }
        __syncthreads();
        for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            int li[10];
#pragma unroll
            for (int l = 0; l < 10; ++l) li[l] = pv.lconn[(int64_t)l * pv.E + e];
            T xe[10 * DPN], ye[10 * DPN];
#pragma unroll
            for (int l = 0; l < 10; ++l)
#pragma unroll
                for (int c = 0; c < DPN; ++c) xe[l * DPN + c] = sx[li[l] * DPN + c];
            K::apply(qd, pv.E, e, cl, cm, xe, ye);
            T d = T(0);
#pragma unroll
            for (int k = 0; k < 10 * DPN; ++k) d += xe[k] * ye[k];
            dot += (double)d;
#pragma unroll
            for (int l = 0; l < 10; ++l)
#pragma unroll
                for (int c = 0; c < DPN; ++c) atomicAdd(&sy[li[l] * DPN + c], ye[l * DPN + c]);
        }
        __syncthreads();
        for (int u = threadIdx.x; u < nloc; u += blockDim.x) {
            const int node = u < nown ? o0 + u : pv.foreign[f0 + u - nown];
            const uint8_t fl = pv.flags[node];
            const bool plain = u < nown && !(fl & kFlagShared);
#pragma unroll
            for (int c = 0; c < DPN; ++c) {
                if ((fl >> c) & 1) continue;
                const T v = sy[u * DPN + c];
                T* dst = y + (int64_t)node * DPN + c;
                if (plain) *dst = v;
                else atomicAdd(dst, v);
            }
        }
        __syncthreads();
    }
    return dot;
}

struct MfArgs {
    PatchView pv;
    const double* qd64;
    const float* qd32;
    double cl, cm, cd;
    int64_t ndof;
    const double* b;          // right-hand side, patch numbering
    double* x64;              // solution (FP64)
    double *r64, *p64, *q64;  // FP64 mode vectors
    const double* dinv64;
    float *xs, *r32, *p32, *q32;  // MIXED inner vectors
    const float* dinv32;
    double* w64;  // MIXED: K x64, then b - K x64
    double *part_a, *part_b, *part_c;
    GridSync* gs;
    PcgResult* res;
    unsigned long long timeout_ns;
    long long max_it;
    double tol, abs_tol, delta;
};

#define MF_BARRIER()                                   \
    do {                                               \
        if (!grid_barrier(a.gs, nb, a.timeout_ns)) return; \
    } while (0)

// Persistent Jacobi-PCG over the matrix-free operator.
//  FP64: the reference loop (iterative.rs:46-119) with its stopping rule on the
//        recursive residual.
//  MIXED: the same loop on FP32 vectors with the FP32 operator; x accumulates
//        in FP32 (xs) and is flushed into the FP64 solution whenever the FP32
//        residual fell by `delta` since the last refresh, at which point the
//        true residual b - K x is recomputed in FP64, the FP32 residual is
//        replaced by it (rescaled to unit norm) and the search direction is kept.
//        Convergence is decided on that FP64 residual.
template <class K64, class K32, bool MIXED>
__global__ void __launch_bounds__(kMfBS) k_mf_pcg(MfArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int DPN = K64::DPN;
    using T = typename std::conditional<MIXED, float, double>::type;
    using KT = typename std::conditional<MIXED, K32, K64>::type;
    const unsigned nb = gridDim.x;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t n = a.ndof;
    const uint8_t* flags = a.pv.flags;
    const double cd = a.cd;
    T* xv = MIXED ? (T*)a.xs : (T*)a.x64;
    T* rv = MIXED ? (T*)a.r32 : (T*)a.r64;
    T* pv = MIXED ? (T*)a.p32 : (T*)a.p64;
    T* qv = MIXED ? (T*)a.q32 : (T*)a.q64;
    const T* dv = MIXED ? (const T*)a.dinv32 : (const T*)a.dinv64;
    const T* qd = MIXED ? (const T*)a.qd32 : (const T*)a.qd64;

    double bnorm, rz, s_scale = 1.0;
    double pdd = 0.0;  // this block's sum of p_i^2 over Dirichlet rows
    {
        double v[2] = {0.0, 0.0};
        for (int64_t i = tid; i < n; i += nth) {
            const double bi = a.b[i];
            v[0] += bi * bi;
            if (!MIXED) {
                const double zi = bi * a.dinv64[i];
                a.x64[i] = 0.0;
                a.r64[i] = bi;
                a.p64[i] = zi;
                v[1] += bi * zi;
                if ((flags[i / DPN] >> (i % DPN)) & 1) pdd += zi * zi;
            } else {
                a.x64[i] = 0.0;
                a.xs[i] = 0.0f;
            }
        }
        store_partial<2>(a.part_b, v);
    }
    MF_BARRIER();
    {
        double t[2];
        grid_total<2>(a.part_b, nb, t);
        bnorm = sqrt(t[0]);
        rz = t[1];
    }
    if (bnorm < 1e-25) {
        if (tid == 0) *a.res = PcgResult{0, 0.0, bnorm, 1, 0, 0};
        return;
    }
    if (MIXED) {
        s_scale = bnorm;
        double v[1] = {0.0};
        const double inv = 1.0 / s_scale;
        for (int64_t i = tid; i < n; i += nth) {
            const float ri = (float)(a.b[i] * inv);
            const float zi = ri * a.dinv32[i];
            a.r32[i] = ri;
            a.p32[i] = zi;
            v[0] += (double)(ri * zi);
            if ((flags[i / DPN] >> (i % DPN)) & 1) pdd += (double)(zi * zi);
        }
        store_partial<1>(a.part_c, v);
        MF_BARRIER();
        double t[1];
        grid_total<1>(a.part_c, nb, t);
        rz = t[0];
    }
    long long it = 0, nupd = 0;
    int converged = 0, breakdown = 0;
    double final_res = bnorm, rmax = 1.0;
    while (it < a.max_it) {
        // ---- q = K_bc p (free rows by elements; Dirichlet rows folded in below)
        {
            double v[1];
            v[0] = element_phase<KT, T>(a.pv, qd, (T)a.cl, (T)a.cm, pv, qv, smem, MODE_FREE);
            v[0] += cd * pdd;
            store_partial<1>(a.part_a, v);
        }
        MF_BARRIER();
        double pq[1];
        grid_total<1>(a.part_a, nb, pq);
        if (fabs(pq[0]) < 1e-30) {
            breakdown = 1;
            break;
        }
        const T alpha = (T)(rz / pq[0]);
        {
            T acc_rr = T(0), acc_rz = T(0);
            for (int64_t i = tid; i < n; i += nth) {
                const uint8_t fl = flags[i / DPN];
                const bool dir = (fl >> (i % DPN)) & 1;
                const T pi = pv[i];
                T qi;
                if (dir) {
                    qi = (T)cd * pi;
                } else {
                    qi = qv[i];
                    if (fl & kFlagShared) qv[i] = T(0);
                }
                xv[i] += alpha * pi;
                const T ri = rv[i] - alpha * qi;
                rv[i] = ri;
                acc_rr += ri * ri;
                acc_rz += ri * (ri * dv[i]);
            }
            double v[2] = {(double)acc_rr, (double)acc_rz};
            store_partial<2>(a.part_b, v);
        }
        MF_BARRIER();
        double t2[2];
        grid_total<2>(a.part_b, nb, t2);
        double rz_new = t2[1];
        const double rn = sqrt(t2[0]);
        if (!MIXED) {
            final_res = rn;
            if (rn < a.tol * bnorm || rn < a.abs_tol) {
                converged = 1;
                break;
            }
        } else {
            rmax = fmax(rmax, rn);
            const double est = rn * s_scale;
            if (est < a.tol * bnorm || est < a.abs_tol || rn < a.delta * rmax) {
                // ---- refresh: x64 += s xs, xs = 0
                for (int64_t i = tid; i < n; i += nth) {
                    a.x64[i] += s_scale * (double)a.xs[i];
                    a.xs[i] = 0.0f;
                }
                MF_BARRIER();
                // ---- w = K_bc x64 (FP64 operator)
                element_phase<K64, double>(a.pv, a.qd64, a.cl, a.cm, a.x64, a.w64, smem, MODE_FREE);
                MF_BARRIER();
                // ---- w = b - K_bc x64 and its norm
                {
                    double v[1] = {0.0};
                    for (int64_t i = tid; i < n; i += nth) {
                        const bool dir = (flags[i / DPN] >> (i % DPN)) & 1;
                        const double kx = dir ? cd * a.x64[i] : a.w64[i];
                        const double ri = a.b[i] - kx;
                        a.w64[i] = ri;
                        v[0] += ri * ri;
                    }
                    store_partial<1>(a.part_c, v);
                }
                MF_BARRIER();
                double t1[1];
                grid_total<1>(a.part_c, nb, t1);
                const double s_new = sqrt(t1[0]);
                ++nupd;
                final_res = s_new;
                if (s_new < a.tol * bnorm || s_new < a.abs_tol) {
                    converged = 1;
                    break;
                }
                // ---- r32 = (b - K x64) / s_new, p32 rescaled, rz recomputed
                {
                    const double ratio = s_scale / s_new, inv = 1.0 / s_new;
                    double v[1] = {0.0};
                    for (int64_t i = tid; i < n; i += nth) {
                        const uint8_t fl = flags[i / DPN];
                        const double wi = a.w64[i];
                        if (!((fl >> (i % DPN)) & 1) && (fl & kFlagShared)) a.w64[i] = 0.0;
                        const float ri = (float)(wi * inv);
                        a.r32[i] = ri;
                        a.p32[i] = (float)((double)a.p32[i] * ratio);
                        v[0] += (double)(ri * (ri * a.dinv32[i]));
                    }
                    store_partial<1>(a.part_a, v);
                    MF_BARRIER();
                    double t1b[1];
                    grid_total<1>(a.part_a, nb, t1b);
                    rz *= ratio * ratio;
                    rz_new = t1b[0];
                    s_scale = s_new;
                    rmax = 1.0;
                }
            }
        }
        const T beta = (T)(rz_new / rz);
        rz = rz_new;
        pdd = 0.0;
        for (int64_t i = tid; i < n; i += nth) {
            const T pnew = rv[i] * dv[i] + beta * pv[i];
            pv[i] = pnew;
            if ((flags[i / DPN] >> (i % DPN)) & 1) pdd += (double)(pnew * pnew);
        }
        MF_BARRIER();
        ++it;
    }
    if (MIXED && !converged) {
        for (int64_t i = tid; i < n; i += nth) {
            a.x64[i] += s_scale * (double)a.xs[i];
            a.xs[i] = 0.0f;
        }
    }
    if (tid == 0) *a.res = PcgResult{it, final_res, bnorm, converged, breakdown, nupd};
}

// ------------------------------------------------------------------ stand-alone kernels
template <class K, class T>
__global__ void __launch_bounds__(kMfBS) k_mf_apply(PatchView pv, const T* qd, T cl, T cm, const T* x, T* y,
                                                     int mode) {
    extern __shared__ __align__(16) unsigned char smem[];
    element_phase<K, T>(pv, qd, cl, cm, x, y, smem, mode);
}

// y_D = cd x_D (MODE_FREE) for the Dirichlet rows after an element pass
template <class T>
__global__ void k_dir_rows(const uint8_t* flags, int dpn, int64_t n, double cd, const T* x, T* y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if ((flags[i / dpn] >> (i % dpn)) & 1) y[i] = (T)(cd * (double)x[i]);
}

// f_bc: free rows f - (K_{F,D} g), Dirichlet rows g cd
__global__ void k_lift_finish(const uint8_t* flags, int dpn, int64_t n, double cd, const double* f,
                              const double* g, const double* kg, double* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool dir = (flags[i / dpn] >> (i % dpn)) & 1;
        out[i] = dir ? g[i] * cd : f[i] - kg[i];
    }
}

template <class T>
__global__ void k_zero_dir(const uint8_t* flags, int dpn, int64_t n, T* v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if ((flags[i / dpn] >> (i % dpn)) & 1) v[i] = T(0);
}

// out[new] = in[orig] / out[orig] = in[new] for interleaved dpn vectors
template <class Tin, class Tout>
__global__ void k_to_new(const int32_t* nperm, int dpn, int64_t N, const Tin* in, Tout* out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * dpn; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / dpn;
        const int c = (int)(t % dpn);
        out[t] = (Tout)in[(int64_t)nperm[i] * dpn + c];
    }
}
template <class Tin, class Tout>
__global__ void k_to_orig(const int32_t* nperm, int dpn, int64_t N, const Tin* in, Tout* out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * dpn; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / dpn;
        const int c = (int)(t % dpn);
        out[(int64_t)nperm[i] * dpn + c] = (Tout)in[t];
    }
}

// ------------------------------------------------------------------ set-up kernels
__device__ __forceinline__ void load_elem(const double* __restrict__ xyz, const int32_t* __restrict__ conn,
                                          int64_t N, int64_t E, int64_t e, double (&X)[10][3]) {
#pragma unroll
    for (int l = 0; l < 10; ++l) {
        const int64_t nd = conn[l * E + e];
        X[l][0] = xyz[nd];
        X[l][1] = xyz[N + nd];
        X[l][2] = xyz[2 * N + nd];
    }
}

// flags[0] |= 1 when some element is not affine (a midpoint off its edge centre)
__global__ void k_affine_check(const double* xyz, const int32_t* conn, int64_t N, int64_t E, int* flag) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    double X[10][3];
    load_elem(xyz, conn, N, E, e, X);
    double h = 0.0;
    for (int k = 0; k < 6; ++k)
        for (int c = 0; c < 3; ++c) h = fmax(h, fabs(X[edge_v(k, 1)][c] - X[edge_v(k, 0)][c]));
    for (int k = 0; k < 6; ++k)
        for (int c = 0; c < 3; ++c) {
            const double mid = 0.5 * (X[edge_v(k, 0)][c] + X[edge_v(k, 1)][c]);
            if (fabs(X[4 + k][c] - mid) > 1e-13 * h) atomicOr(flag, 1);
        }
}

// geometry at QP q (NQ == 4) or the affine vertex Jacobian (NQ == 1)
template <int NQ>
__device__ __forceinline__ void elem_jacobian(const double (&X)[10][3], int q, double (&J)[3][3]) {
    if (NQ == 1) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) J[r][c] = X[c + 1][r] - X[0][r];
    } else {
        double L[4];
        qp4(q, L);
        jacobian10(X, L, J);
    }
}

// qdata in patch element order (see matfree.cuh)
template <int NQ>
__global__ void k_qdata(int phys, const double* xyz, const int32_t* conn, const int32_t* eperm, int64_t N,
                        int64_t E, const double* coef, double* qd64, float* qd32, int* err) {
    const int64_t ne = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (ne >= E) return;
    const int64_t e = eperm[ne];
    double X[10][3];
    load_elem(xyz, conn, N, E, e, X);
    const double k = coef[e];
    for (int q = 0; q < NQ; ++q) {
        double J[3][3], A[3][3];
        elem_jacobian<NQ>(X, q, J);
        const double d = det3(J);
        if (d == 0.0) {
            atomicOr(err, DEV_ERR_SINGULAR);
            return;
        }
        adj3(J, A);
        if (phys == 0) {
            const double s = k * kQw / fabs(d);
            double G[6];
            G[0] = s * (A[0][0] * A[0][0] + A[0][1] * A[0][1] + A[0][2] * A[0][2]);
            G[1] = s * (A[0][0] * A[1][0] + A[0][1] * A[1][1] + A[0][2] * A[1][2]);
            G[2] = s * (A[0][0] * A[2][0] + A[0][1] * A[2][1] + A[0][2] * A[2][2]);
            G[3] = s * (A[1][0] * A[1][0] + A[1][1] * A[1][1] + A[1][2] * A[1][2]);
            G[4] = s * (A[1][0] * A[2][0] + A[1][1] * A[2][1] + A[1][2] * A[2][2]);
            G[5] = s * (A[2][0] * A[2][0] + A[2][1] * A[2][1] + A[2][2] * A[2][2]);
            for (int j = 0; j < 6; ++j) {
                qd64[(6 * q + j) * E + ne] = G[j];
                qd32[(6 * q + j) * E + ne] = (float)G[j];
            }
        } else {
            double v[10];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) v[3 * r + c] = A[r][c] / d;
            v[9] = kQw * fabs(d) * k;
            for (int j = 0; j < 10; ++j) {
                qd64[(10 * q + j) * E + ne] = v[j];
                qd32[(10 * q + j) * E + ne] = (float)v[j];
            }
        }
    }
}

// Diagonal of every K_e, original element order: ediag[e][dpn*l + c].
__global__ void k_ediag(int phys, const double* xyz, const int32_t* conn, int64_t N, int64_t E, const double* coef,
                        double cl, double cm, double* ediag, int* err) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    double X[10][3];
    load_elem(xyz, conn, N, E, e, X);
    const double k = coef[e];
    const int dpn = phys == 0 ? 1 : 3;
    double acc[30];
    for (int i = 0; i < 30; ++i) acc[i] = 0.0;
    for (int q = 0; q < 4; ++q) {
        double L[4], J[3][3], A[3][3];
        qp4(q, L);
        jacobian10(X, L, J);
        const double d = det3(J);
        if (d == 0.0) {
            atomicOr(err, DEV_ERR_SINGULAR);
            return;
        }
        adj3(J, A);
        double Ji[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Ji[r][c] = A[r][c] / d;
        const double w = kQw * fabs(d);
        for (int l = 0; l < 10; ++l) {
            double g[3], gc[3];
            ref_grad(l, L, g);
            cart_grad(Ji, g, gc);
            const double gg = gc[0] * gc[0] + gc[1] * gc[1] + gc[2] * gc[2];
            if (phys == 0) {
                acc[l] += k * gg * w;
            } else {
                for (int c = 0; c < 3; ++c)
                    acc[3 * l + c] += w * k * (cl * gc[c] * gc[c] + cm * (gg + gc[c] * gc[c]));
            }
        }
    }
    for (int i = 0; i < 10 * dpn; ++i) ediag[e * 10 * dpn + i] = acc[i];
}

__global__ void k_gather_diag(const int32_t* ptr, const int32_t* inc, const double* ediag, int64_t N, int dpn,
                              double* diag) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= N * dpn) return;
    const int64_t i = t / dpn;
    const int c = (int)(t % dpn);
    double s = 0.0;
    for (int32_t p = ptr[i]; p < ptr[i + 1]; ++p) {
        const int32_t el = inc[p];
        s += ediag[(int64_t)(el / 10) * 10 * dpn + dpn * (el % 10) + c];
    }
    diag[t] = s;
}

__global__ void k_max_abs(const double* v, int64_t n, unsigned long long* out) {
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(v[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// dinv in patch numbering (JacobiPreconditioner::new, preconditioner.rs:37-51 on K_bc)
__global__ void k_dinv(const int32_t* nperm, const uint8_t* flags, int dpn, int64_t N, const double* diag_orig,
                       double cd, double* d64, float* d32, double* dg_out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * dpn; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / dpn;
        const int c = (int)(t % dpn);
        const bool dir = (flags[i] >> c) & 1;
        const double dd = dir ? cd : diag_orig[(int64_t)nperm[i] * dpn + c];
        const double inv = fabs(dd) > 1e-14 ? 1.0 / dd : 1.0;
        d64[t] = inv;
        d32[t] = (float)inv;
        if (dg_out) dg_out[t] = dd;
    }
}

// Adjoint element gradient g_e = -lambda_e^T K_e u_e (original order, FP64),
// lambda read as zero on Dirichlet DOFs. Isoparametric, so curved elements too.
__global__ void k_elem_gradient(int phys, const double* xyz, const int32_t* conn, int64_t N, int64_t E,
                                const double* coef, double cl, double cm, const uint8_t* mask, const double* u,
                                const double* lam, double* g) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    double X[10][3];
    load_elem(xyz, conn, N, E, e, X);
    const double k = coef[e];
    const int dpn = phys == 0 ? 1 : 3;
    double ue[30], le[30];
    for (int l = 0; l < 10; ++l) {
        const int64_t nd = conn[l * E + e];
        for (int c = 0; c < dpn; ++c) {
            const int64_t dof = nd * dpn + c;
            ue[l * dpn + c] = u[dof];
            le[l * dpn + c] = mask[dof] ? 0.0 : lam[dof];
        }
    }
    double s = 0.0;
    for (int q = 0; q < 4; ++q) {
        double L[4], J[3][3], A[3][3];
        qp4(q, L);
        jacobian10(X, L, J);
        const double d = det3(J);
        if (d == 0.0) continue;
        adj3(J, A);
        double Ji[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Ji[r][c] = A[r][c] / d;
        const double w = kQw * fabs(d);
        double Fu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Fl[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int l = 0; l < 10; ++l) {
            double gr[3], gc[3];
            ref_grad(l, L, gr);
            cart_grad(Ji, gr, gc);
            for (int c = 0; c < dpn; ++c)
                for (int b = 0; b < 3; ++b) {
                    Fu[c][b] += ue[l * dpn + c] * gc[b];
                    Fl[c][b] += le[l * dpn + c] * gc[b];
                }
        }
        if (phys == 0) {
            s += k * w * (Fu[0][0] * Fl[0][0] + Fu[0][1] * Fl[0][1] + Fu[0][2] * Fl[0][2]);
        } else {
            const double tu = Fu[0][0] + Fu[1][1] + Fu[2][2], tl = Fl[0][0] + Fl[1][1] + Fl[2][2];
            double ee = 0.0;
            for (int c = 0; c < 3; ++c)
                for (int b = 0; b < 3; ++b) ee += 0.5 * (Fu[c][b] + Fu[b][c]) * (Fl[c][b] + Fl[b][c]);
            // lambda tr(eps_u) tr(eps_l) + 2 mu eps_u : eps_l, with lambda = k cl, mu = k cm
            s += w * k * (cl * tu * tl + cm * ee);
        }
    }
    g[e] = -s;
}

}  // namespace geo

// ====================================================================== operator object
struct geo_op {
    geo_ctx* ctx = nullptr;
    const geo_mesh* mesh = nullptr;
    int phys = 0, dpn = 1, nq = 1;
    int64_t N = 0, E = 0, ndof = 0;
    int n_patches = 0, ucap = 0;
    double nu = 0, cl = 0, cm = 0, cd = 1.0, coef_scalar = 1.0;
    geo::DevBuf<int32_t> eperm, nperm, pe, po, pf, foreign;
    geo::DevBuf<uint16_t> lconn;
    geo::DevBuf<uint8_t> flags;
    geo::DevBuf<uint8_t> mask_orig;  // Dirichlet mask, original DOF numbering
    geo::DevBuf<double> coef, qd64, g_new, diag_new, dinv64, ediag, diag_orig;
    geo::DevBuf<float> qd32, dinv32;
    // solver workspace
    geo::DevBuf<double> w64;
    geo::DevBuf<float> w32;
    geo::PcgScratch sc;
    int pcg_blocks[2][2] = {{0, 0}, {0, 0}};
};

namespace geo {
namespace {

inline unsigned nblk(int64_t n, int bs = 256) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, bs), 148 * 64));
}

PatchView view(const geo_op* op) {
    PatchView v;
    v.E = op->E;
    v.N = op->N;
    v.n_patches = op->n_patches;
    v.ucap = op->ucap;
    v.dpn = op->dpn;
    v.pe = op->pe.p;
    v.po = op->po.p;
    v.pf = op->pf.p;
    v.foreign = op->foreign.p;
    v.lconn = op->lconn.p;
    v.flags = op->flags.p;
    return v;
}

size_t smem_bytes(const geo_op* op, size_t elt) { return (size_t)2 * op->ucap * op->dpn * elt; }

template <class F>
void with_kernels(const geo_op* op, F&& f) {
    // dispatch (physics, NQ) to concrete element kernels
    if (op->phys == 0) {
        if (op->nq == 1) f(ThermalK<double, 1>{}, ThermalK<float, 1>{});
        else f(ThermalK<double, 4>{}, ThermalK<float, 4>{});
    } else {
        if (op->nq == 1) f(ElasticK<double, 1>{}, ElasticK<float, 1>{});
        else f(ElasticK<double, 4>{}, ElasticK<float, 4>{});
    }
}

template <class K, class T>
void set_smem_attr(size_t bytes) {
    GEO_CUDA(cudaFuncSetAttribute(k_mf_apply<K, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// Recomputes qdata, diagonal, char_diag and the Jacobi inverse from op->coef.
void refresh_coefficients(geo_op* op) {
    geo_ctx* ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    const geo_mesh* m = op->mesh;
    reset_dev_err(ctx);
    const int nqd = (op->phys == 0 ? 6 : 10) * op->nq;
    op->qd64.ensure((size_t)nqd * op->E);
    op->qd32.ensure((size_t)nqd * op->E);
    if (op->nq == 1)
        k_qdata<1><<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->eperm.p, op->N, op->E,
                                                    op->coef.p, op->qd64.p, op->qd32.p, ctx->dev_err.p);
    else
        k_qdata<4><<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->eperm.p, op->N,
                                                              op->E, op->coef.p, op->qd64.p, op->qd32.p,
                                                              ctx->dev_err.p);
    check_launch(ctx, "k_qdata");
    op->ediag.ensure((size_t)op->E * 10 * op->dpn);
    k_ediag<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->N, op->E, op->coef.p,
                                                       op->cl, op->cm, op->ediag.p, ctx->dev_err.p);
    check_launch(ctx, "k_ediag");
    raise_dev_err(ctx, read_dev_err(ctx), "operator set-up");
    op->diag_orig.ensure(op->ndof);
    k_gather_diag<<<(unsigned)cdiv(op->ndof, 256), 256, 0, s>>>(m->inc_ptr.p, m->inc.p, op->ediag.p, op->N,
                                                                op->dpn, op->diag_orig.p);
    check_launch(ctx, "k_gather_diag");
    DevBuf<unsigned long long> mx(1);
    GEO_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(unsigned long long), s));
    k_max_abs<<<nblk(op->ndof), 256, 0, s>>>(op->diag_orig.p, op->ndof, mx.p);
    check_launch(ctx, "k_max_abs");
    unsigned long long bits = 0;
    GEO_CUDA(cudaMemcpyAsync(&bits, mx.p, sizeof(bits), cudaMemcpyDeviceToHost, s));
    sync(ctx, "char_diag");
    double maxd;
    std::memcpy(&maxd, &bits, sizeof(double));
    op->cd = maxd > 1.0 ? maxd : 1.0;  // assembly.rs:184-193
    op->dinv64.ensure(op->ndof);
    op->dinv32.ensure(op->ndof);
    op->diag_new.ensure(op->ndof);
    k_dinv<<<nblk(op->ndof), 256, 0, s>>>(op->nperm.p, op->flags.p, op->dpn, op->N, op->diag_orig.p, op->cd,
                                         op->dinv64.p, op->dinv32.p, op->diag_new.p);
    check_launch(ctx, "k_dinv");
    sync(ctx, "operator coefficients");
}

void set_coef(geo_op* op, const double* coef_e, double coef) {
    cudaStream_t s = op->ctx->stream;
    op->coef.ensure(op->E);
    if (coef_e) {
        GEO_CUDA(cudaMemcpyAsync(op->coef.p, coef_e, op->E * sizeof(double), cudaMemcpyDefault, s));
    } else {
        std::vector<double> h(op->E, coef);
        GEO_CUDA(cudaMemcpyAsync(op->coef.p, h.data(), op->E * sizeof(double), cudaMemcpyHostToDevice, s));
        sync(op->ctx, "coefficients");
    }
    op->coef_scalar = coef;
}

geo_op* create_op(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, int phys, const double* coef_e,
                  double coef, double nu) {
    GEO_CHECK_ARG(ctx && mesh && dofs, "NULL argument");
    GEO_CHECK_ARG(dofs->n_nodes == mesh->n_nodes, "DOF manager and mesh disagree on the node count");
    const int dpn = phys == 0 ? 1 : 3;
    GEO_CHECK_ARG(dofs->dpn == dpn, phys == 0 ? "thermal operator needs 1 DOF per node"
                                              : "Elasticity requires 3 DOF per node");
    auto op = std::make_unique<geo_op>();
    op->ctx = ctx;
    op->mesh = mesh;
    op->phys = phys;
    op->dpn = dpn;
    op->N = mesh->n_nodes;
    op->E = mesh->n_elem;
    op->ndof = op->N * dpn;
    op->nu = nu;
    op->cl = phys == 1 ? nu / ((1.0 + nu) * (1.0 - 2.0 * nu)) : 0.0;
    op->cm = phys == 1 ? 1.0 / (2.0 * (1.0 + nu)) : 0.0;
    cudaStream_t s = ctx->stream;
    ensure_inverse_map(const_cast<geo_mesh*>(mesh));
    PatchLayout L;
    try {
        build_patches(op->N, mesh->h_xyz.data(), op->E, mesh->h_conn.data(), L);
    } catch (const std::exception& ex) {
        fail(GEO_ERR_UNSUPPORTED, ex.what());
    }
    op->n_patches = (int)L.n_patches;
    op->ucap = L.max_local;
    // node flags in patch numbering: Dirichlet bit per component + shared bit
    std::vector<uint8_t> fl(op->N, 0);
    for (int64_t i = 0; i < op->N; ++i) {
        const int64_t o = L.nperm[i];
        uint8_t f = L.shared[i] ? kFlagShared : 0;
        for (int c = 0; c < dpn; ++c)
            if (dofs->h_mask[o * dpn + c]) f |= (uint8_t)(kFlagDir0 << c);
        fl[i] = f;
    }
    std::vector<double> gnew(op->ndof);
    for (int64_t i = 0; i < op->N; ++i)
        for (int c = 0; c < dpn; ++c) gnew[i * dpn + c] = dofs->h_vals[(int64_t)L.nperm[i] * dpn + c];
    auto up = [&](auto& buf, const auto& vec) {
        buf.alloc(std::max<size_t>(vec.size(), 1));
        if (!vec.empty())
            GEO_CUDA(cudaMemcpyAsync(buf.p, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice, s));
    };
    up(op->eperm, L.eperm);
    up(op->nperm, L.nperm);
    up(op->pe, L.patch_elem);
    up(op->po, L.patch_own);
    up(op->pf, L.patch_foreign);
    up(op->foreign, L.foreign);
    up(op->lconn, L.lconn);
    up(op->flags, fl);
    up(op->g_new, gnew);
    up(op->mask_orig, dofs->h_mask);
    sync(ctx, "operator upload");
    // affine (straight-sided) elements use one metric per element
    DevBuf<int> aff(1);
    GEO_CUDA(cudaMemsetAsync(aff.p, 0, sizeof(int), s));
    k_affine_check<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(mesh->xyz.p, mesh->conn.p, op->N, op->E, aff.p);
    check_launch(ctx, "k_affine_check");
    int curved = 0;
    GEO_CUDA(cudaMemcpyAsync(&curved, aff.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    sync(ctx, "affine check");
    op->nq = curved ? 4 : 1;
    set_coef(op.get(), coef_e, coef);
    refresh_coefficients(op.get());
    with_kernels(op.get(), [&](auto k64, auto k32) {
        using K64 = decltype(k64);
        using K32 = decltype(k32);
        set_smem_attr<K64, double>(smem_bytes(op.get(), 8));
        set_smem_attr<K32, float>(smem_bytes(op.get(), 4));
        GEO_CUDA(cudaFuncSetAttribute(k_mf_pcg<K64, K32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem_bytes(op.get(), 8)));
        GEO_CUDA(cudaFuncSetAttribute(k_mf_pcg<K64, K32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem_bytes(op.get(), 8)));
        op->pcg_blocks[0][0] = persistent_blocks(ctx, k_mf_pcg<K64, K32, false>, kMfBS, smem_bytes(op.get(), 8));
        op->pcg_blocks[0][1] = persistent_blocks(ctx, k_mf_pcg<K64, K32, true>, kMfBS, smem_bytes(op.get(), 8));
    });
    return op.release();
}

// y = K_bc x in patch numbering (device vectors of type T)
template <class T>
void apply_new(geo_op* op, const T* x, T* y, int mode) {
    geo_ctx* ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    GEO_CUDA(cudaMemsetAsync(y, 0, op->ndof * sizeof(T), s));
    const PatchView pv = view(op);
    with_kernels(op, [&](auto k64, auto k32) {
        using K = typename std::conditional<std::is_same<T, double>::value, decltype(k64), decltype(k32)>::type;
        const T* qd = std::is_same<T, double>::value ? (const T*)op->qd64.p : (const T*)op->qd32.p;
        k_mf_apply<K, T><<<(unsigned)op->n_patches, kMfBS, smem_bytes(op, sizeof(T)), s>>>(
            pv, qd, (T)op->cl, (T)op->cm, x, y, mode);
    });
    check_launch(ctx, "k_mf_apply");
    if (mode == MODE_FREE) {
        k_dir_rows<T><<<nblk(op->ndof), 256, 0, s>>>(op->flags.p, op->dpn, op->ndof, op->cd, x, y);
        check_launch(ctx, "k_dir_rows");
    }
}

void to_new(geo_op* op, const double* in_orig, double* out_new) {
    k_to_new<double, double><<<nblk(op->ndof), 256, 0, op->ctx->stream>>>(op->nperm.p, op->dpn, op->N, in_orig,
                                                                          out_new);
    check_launch(op->ctx, "k_to_new");
}
void to_orig(geo_op* op, const double* in_new, double* out_orig) {
    k_to_orig<double, double><<<nblk(op->ndof), 256, 0, op->ctx->stream>>>(op->nperm.p, op->dpn, op->N, in_new,
                                                                           out_orig);
    check_launch(op->ctx, "k_to_orig");
}

// f_bc (patch numbering) from f (original numbering), device buffers
void lift_new(geo_op* op, const double* f_orig_dev, double* fbc_new) {
    cudaStream_t s = op->ctx->stream;
    DevBuf<double> fn(op->ndof), kg(op->ndof);
    to_new(op, f_orig_dev, fn.p);
    apply_new<double>(op, op->g_new.p, kg.p, MODE_LIFT);
    k_lift_finish<<<nblk(op->ndof), 256, 0, s>>>(op->flags.p, op->dpn, op->ndof, op->cd, fn.p, op->g_new.p, kg.p,
                                                fbc_new);
    check_launch(op->ctx, "k_lift_finish");
    sync(op->ctx, "lift");
}

// Persistent PCG on K_bc; b_new / x_new in patch numbering (device).
int solve_new(geo_op* op, const double* b_new, const geo_cg_opts& o, double* x_new, geo_solver_stats* st) {
    geo_ctx* ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    const bool mixed = o.precision == GEO_PRECISION_MIXED;
    const int64_t n = op->ndof;
    int nb = op->pcg_blocks[0][mixed ? 1 : 0];
    op->sc.ensure(nb);
    // workspace: FP64 r, p, q (FP64 mode) or w (mixed); FP32 xs, r, p, q (mixed)
    op->w64.ensure((size_t)3 * n);
    if (mixed) op->w32.ensure((size_t)4 * n);
    MfArgs a{};
    a.pv = view(op);
    a.qd64 = op->qd64.p;
    a.qd32 = op->qd32.p;
    a.cl = op->cl;
    a.cm = op->cm;
    a.cd = op->cd;
    a.ndof = n;
    a.b = b_new;
    a.x64 = x_new;
    a.r64 = op->w64.p;
    a.p64 = op->w64.p + n;
    a.q64 = op->w64.p + 2 * n;
    a.w64 = op->w64.p;
    a.dinv64 = op->dinv64.p;
    a.dinv32 = op->dinv32.p;
    if (mixed) {
        a.xs = op->w32.p;
        a.r32 = op->w32.p + n;
        a.p32 = op->w32.p + 2 * n;
        a.q32 = op->w32.p + 3 * n;
        GEO_CUDA(cudaMemsetAsync(a.q32, 0, n * sizeof(float), s));
        GEO_CUDA(cudaMemsetAsync(a.w64, 0, n * sizeof(double), s));
    } else {
        GEO_CUDA(cudaMemsetAsync(a.q64, 0, n * sizeof(double), s));
    }
    a.part_a = op->sc.slot(0, nb);
    a.part_b = op->sc.slot(1, nb);
    a.part_c = op->sc.slot(2, nb);
    a.gs = op->sc.gs.p;
    a.res = op->sc.res.p;
    a.timeout_ns = (unsigned long long)(o.timeout_seconds * 1e9);
    a.max_it = o.max_iterations;
    a.tol = o.tolerance;
    a.abs_tol = o.abs_tolerance;
    a.delta = o.reliable_delta;
    GEO_CHECK_ARG(o.use_preconditioner, "the matrix-free solver is Jacobi-preconditioned only");
    GEO_CUDA(cudaMemsetAsync(op->sc.gs.p, 0, sizeof(GridSync), s));
    GEO_CUDA(cudaMemsetAsync(op->sc.res.p, 0, sizeof(PcgResult), s));
    const size_t smem = smem_bytes(op, 8);
    GEO_CUDA(cudaEventRecord(ctx->ev0, s));
    with_kernels(op, [&](auto k64, auto k32) {
        using K64 = decltype(k64);
        using K32 = decltype(k32);
        if (mixed) launch_persistent(ctx, k_mf_pcg<K64, K32, true>, kMfBS, smem, a, nb);
        else launch_persistent(ctx, k_mf_pcg<K64, K32, false>, kMfBS, smem, a, nb);
    });
    GEO_CUDA(cudaEventRecord(ctx->ev1, s));
    PcgResult r{};
    GridSync g{};
    GEO_CUDA(cudaMemcpyAsync(&r, op->sc.res.p, sizeof(r), cudaMemcpyDeviceToHost, s));
    GEO_CUDA(cudaMemcpyAsync(&g, op->sc.gs.p, sizeof(g), cudaMemcpyDeviceToHost, s));
    sync(ctx, "matrix-free PCG");
    float ms = 0.f;
    GEO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (g.error & DEV_ERR_TIMEOUT) {
        fill_stats(st, r, ms * 1e-3, GEO_ERR_TIMEOUT);
        fail(GEO_ERR_TIMEOUT, "PCG grid barrier timed out");
    }
    const int status = r.converged ? GEO_OK : (r.breakdown ? GEO_ERR_BREAKDOWN : GEO_NOT_CONVERGED);
    fill_stats(st, r, ms * 1e-3, status);
    return status;
}

int finish_status(geo_ctx* ctx, int status) {
    if (status != GEO_OK)
        record_error(ctx, status, status == GEO_ERR_BREAKDOWN ? "CG breakdown: |p^T A p| < 1e-30"
                                                              : "CG did not converge");
    return status;
}

// ---- failure-detection test kernel: block 0 leaves without arriving
__global__ void k_barrier_probe(GridSync* gs, unsigned long long timeout_ns) {
    if (blockIdx.x == 0) return;
    grid_barrier(gs, gridDim.x, timeout_ns);
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

int geo_thermal_operator_create(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, const double* k_e,
                                double k, geo_op** out) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(out, "out is NULL");
    *out = create_op(ctx, mesh, dofs, 0, k_e, k, 0.0);
    GEO_API_END
}

int geo_elasticity_operator_create(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, const double* E_e,
                                   double E, double nu, geo_op** out) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(out, "out is NULL");
    GEO_CHECK_ARG(nu > -1.0 && nu < 0.5, "Poisson's ratio must be in (-1, 0.5)");
    *out = create_op(ctx, mesh, dofs, 1, E_e, E, nu);
    GEO_API_END
}

int geo_op_set_coefficients(geo_op* op, const double* coef_e, double coef) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op, "NULL operator");
    set_coef(op, coef_e, coef);
    refresh_coefficients(op);
    GEO_API_END
}

int geo_op_info(const geo_op* op, int64_t* n_dofs, int64_t* n_elem, double* char_diag) {
    if (!op) return GEO_ERR_INVALID_ARG;
    if (n_dofs) *n_dofs = op->ndof;
    if (n_elem) *n_elem = op->E;
    if (char_diag) *char_diag = op->cd;
    return GEO_OK;
}

int geo_op_apply(geo_op* op, const double* x, double* y, int32_t precision) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && x && y, "NULL argument");
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    DevBuf<double> tx, xn(n), yn(n), yo(n);
    const double* dx = stage_in(x, n, tx, s);
    to_new(op, dx, xn.p);
    if (precision == GEO_PRECISION_MIXED) {
        DevBuf<float> x32(n), y32(n);
        k_to_new<double, float><<<nblk(n), 256, 0, s>>>(op->nperm.p, op->dpn, op->N, dx, x32.p);
        apply_new<float>(op, x32.p, y32.p, MODE_FREE);
        k_to_orig<float, double><<<nblk(n), 256, 0, s>>>(op->nperm.p, op->dpn, op->N, y32.p, yo.p);
        check_launch(op->ctx, "k_to_orig");
        copy_out(y, yo.p, n, s);
        sync(op->ctx, "geo_op_apply");
    } else {
        apply_new<double>(op, xn.p, yn.p, MODE_FREE);
        to_orig(op, yn.p, yo.p);
        copy_out(y, yo.p, n, s);
        sync(op->ctx, "geo_op_apply");
    }
    GEO_API_END
}

int geo_op_lift_rhs(geo_op* op, const double* f, double* f_bc) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && f && f_bc, "NULL argument");
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    DevBuf<double> tf, fb(n), fo(n);
    const double* df = stage_in(f, n, tf, s);
    lift_new(op, df, fb.p);
    to_orig(op, fb.p, fo.p);
    copy_out(f_bc, fo.p, n, s);
    sync(op->ctx, "geo_op_lift_rhs");
    GEO_API_END
}

int geo_op_diagonal(geo_op* op, double* diag) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && diag, "NULL argument");
    DevBuf<double> d(op->ndof);
    to_orig(op, op->diag_new.p, d.p);
    copy_out(diag, d.p, op->ndof, op->ctx->stream);
    sync(op->ctx, "geo_op_diagonal");
    GEO_API_END
}

int geo_cg_solve_matfree(geo_op* op, const double* b, const geo_cg_opts* opts, double* x, geo_solver_stats* st) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && b && x, "NULL argument");
    geo_cg_opts o;
    cg_opts_fill(opts, o);
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    DevBuf<double> tb, bn(n), xn(n), xo(n);
    const double* db = stage_in(b, n, tb, s);
    to_new(op, db, bn.p);
    const int status = solve_new(op, bn.p, o, xn.p, st);
    to_orig(op, xn.p, xo.p);
    copy_out(x, xo.p, n, s);
    sync(op->ctx, "geo_cg_solve_matfree");
    return finish_status(op->ctx, status);
    GEO_API_END
}

int geo_op_element_gradient(geo_op* op, const double* u, const double* lambda, double* grad_e) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && u && lambda && grad_e, "NULL argument");
    cudaStream_t s = op->ctx->stream;
    DevBuf<double> tu, tl, g(op->E);
    const double* du = stage_in(u, op->ndof, tu, s);
    const double* dl = stage_in(lambda, op->ndof, tl, s);
    const geo_mesh* m = op->mesh;
    k_elem_gradient<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->N, op->E,
                                                               op->coef.p, op->cl, op->cm, op->mask_orig.p, du, dl,
                                                               g.p);
    check_launch(op->ctx, "k_elem_gradient");
    copy_out(grad_e, g.p, op->E, s);
    sync(op->ctx, "geo_op_element_gradient");
    GEO_API_END
}

int geo_forward(geo_op* op, const double* f, const geo_cg_opts* opts, double* u, geo_solver_stats* st) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && f && u, "NULL argument");
    geo_cg_opts o;
    cg_opts_fill(opts, o);
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    DevBuf<double> tf, fb(n), xn(n), xo(n);
    const double* df = stage_in(f, n, tf, s);
    lift_new(op, df, fb.p);
    const int status = solve_new(op, fb.p, o, xn.p, st);
    to_orig(op, xn.p, xo.p);
    copy_out(u, xo.p, n, s);
    sync(op->ctx, "geo_forward");
    return finish_status(op->ctx, status);
    GEO_API_END
}

int geo_vjp(geo_op* op, const double* f, const double* u, const double* dJ_du, const geo_cg_opts* opts,
            double* dJ_dlncoef, geo_solver_stats* st) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && dJ_du && dJ_dlncoef && (u || f), "NULL argument");
    geo_cg_opts o;
    cg_opts_fill(opts, o);
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    DevBuf<double> tu, tg, uo(n), gn(n), ln(n), lo(n), ge(op->E);
    const double* du = nullptr;
    if (u) {
        du = stage_in(u, n, tu, s);
    } else {
        // recompute the forward solution instead of storing it
        DevBuf<double> tf, fb(n), xn(n);
        const double* df = stage_in(f, n, tf, s);
        lift_new(op, df, fb.p);
        const int fs = solve_new(op, fb.p, o, xn.p, nullptr);
        if (fs != GEO_OK) return finish_status(op->ctx, fs);
        to_orig(op, xn.p, uo.p);
        du = uo.p;
    }
    // adjoint right-hand side: dJ/du on free DOFs, zero on Dirichlet DOFs (K_bc
    // is symmetric and its Dirichlet rows are decoupled, so lambda_D = 0)
    const double* dg = stage_in(dJ_du, n, tg, s);
    to_new(op, dg, gn.p);
    k_zero_dir<double><<<nblk(n), 256, 0, s>>>(op->flags.p, op->dpn, n, gn.p);
    check_launch(op->ctx, "adjoint rhs");
    const int status = solve_new(op, gn.p, o, ln.p, st);
    to_orig(op, ln.p, lo.p);
    const geo_mesh* m = op->mesh;
    k_elem_gradient<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->N, op->E,
                                                               op->coef.p, op->cl, op->cm, op->mask_orig.p, du,
                                                               lo.p, ge.p);
    check_launch(op->ctx, "k_elem_gradient");
    copy_out(dJ_dlncoef, ge.p, op->E, s);
    sync(op->ctx, "geo_vjp");
    return finish_status(op->ctx, status);
    GEO_API_END
}

int geo_op_destroy(geo_op* op) {
    if (!op) return GEO_OK;
    cudaSetDevice(op->ctx->device);
    cudaStreamSynchronize(op->ctx->stream);
    delete op;
    return GEO_OK;
}

int geo_debug_barrier_timeout(geo_ctx* ctx, double timeout_seconds) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx, "NULL context");
    GEO_CHECK_ARG(timeout_seconds > 0 && timeout_seconds <= 5.0, "timeout must be in (0, 5] seconds");
    DevBuf<GridSync> gs(1);
    GEO_CUDA(cudaMemsetAsync(gs.p, 0, sizeof(GridSync), ctx->stream));
    const int nb = std::min(persistent_blocks(ctx, k_barrier_probe, 128, 0), 2 * ctx->sm_count);
    GridSync* gp = gs.p;
    unsigned long long tns = (unsigned long long)(timeout_seconds * 1e9);
    void* params[] = {&gp, &tns};
    GEO_CUDA(cudaLaunchCooperativeKernel((const void*)k_barrier_probe, dim3(nb), dim3(128), params, 0, ctx->stream));
    GridSync g{};
    GEO_CUDA(cudaMemcpyAsync(&g, gs.p, sizeof(g), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx, "barrier probe");
    if (g.error & DEV_ERR_TIMEOUT) fail(GEO_ERR_TIMEOUT, "device-side grid barrier timed out (as the probe intends)");
    GEO_API_END
}

}  // extern "C"
