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
// red.global.add for the shared ones (so the matrix-free apply is not
// bit-reproducible in the last bit; the assembled path is). The PCG of the
// operator runs in halo mode instead: foreign contributions are stored to
// per-entry slots and added by the node update in slot order, with no atomics.
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <type_traits>

#include <cub/cub.cuh>

#include "mf_kernels.cuh"
#include "pcg_common.cuh"

struct geo_op;

namespace geo {

// f_bc: free rows f - (K_{F,D} g), Dirichlet rows g cd
__global__ void k_lift_finish(const uint8_t* flags, int dpn, int64_t n, double cd, const double* f,
                              const double* g, const double* kg, double* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool dir = (flags[i / dpn] >> (i % dpn)) & 1;
        out[i] = dir ? g[i] * cd : f[i] - kg[i];
    }
}

__global__ void k_scale(double* v, int64_t n, double a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] *= a;
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
// node flags (Dirichlet bits, shared bit) and Dirichlet values in patch numbering
__global__ void k_node_flags(const int32_t* nperm, const uint8_t* shared, const uint8_t* mask, const double* vals,
                             int dpn, int64_t N, uint8_t* flags, double* g_new) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = nperm[i];
        uint8_t f = shared[i] ? kFlagShared : 0;
        for (int c = 0; c < dpn; ++c) {
            if (mask[o * dpn + c]) f |= (uint8_t)(kFlagDir0 << c);
            g_new[i * dpn + c] = vals[o * dpn + c];
        }
        flags[i] = f;
    }
}

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
                const int64_t at = ((ne / kPatchElems) * (6 * NQ) + 6 * q + j) * kPatchElems + ne % kPatchElems;
                qd64[at] = G[j];
                qd32[at] = (float)G[j];
            }
        } else {
            double v[10];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) v[3 * r + c] = A[r][c] / d;
            v[9] = kQw * fabs(d) * k;
            for (int j = 0; j < 10; ++j) {
                const int64_t at = ((ne / kPatchElems) * (10 * NQ) + 10 * q + j) * kPatchElems + ne % kPatchElems;
                qd64[at] = v[j];
                qd32[at] = (float)v[j];
            }
        }
    }
}

// Foreign ids and flags of every patch copied into segments that start at
// pfa[p] (multiples of kForeignAlign entries), so that the patch kernel's bulk
// copy brings them with the element data. One block per patch.
__global__ void k_patch_foreign(const int32_t* __restrict__ pf, const int32_t* __restrict__ pfa,
                               const int32_t* __restrict__ foreign, const uint8_t* __restrict__ flags,
                               int32_t* __restrict__ fids, uint8_t* __restrict__ fflags) {
    const int p = blockIdx.x;
    const int f0 = pf[p], nf = pf[p + 1] - f0, a0 = pfa[p];
    for (int k = threadIdx.x; k < nf; k += blockDim.x) {
        const int32_t nd = foreign[f0 + k];
        fids[a0 + k] = nd;
        fflags[a0 + k] = flags[nd];
    }
}

// Halo slots of the PCG (thermal and elasticity): every foreign entry a (patch p, its
// k-th foreign node n, a = pf[p] + k) gets a slot. Slots are ordered by node n,
// then by entry (a stable sort of the entries by node), so node n's slots are
// consecutive and follow those of the nodes before it.
__global__ void k_halo_count(const int32_t* __restrict__ foreign, int64_t n_app, int32_t* __restrict__ cnt) {
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < n_app; a += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[foreign[a]], 1);
}
__global__ void k_iota(int64_t n, int32_t* __restrict__ v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = (int32_t)i;
}
__global__ void k_halo_slot_of(const int32_t* __restrict__ sorted_app, int64_t n_app, int32_t* __restrict__ slot_of) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_app; t += (int64_t)gridDim.x * blockDim.x)
        slot_of[sorted_app[t]] = (int32_t)t;
}
// the slots again in the per-patch segments of fids (one block per patch)
__global__ void k_patch_fslot(const int32_t* __restrict__ pf, const int32_t* __restrict__ pfa,
                              const int32_t* __restrict__ slot_of, int32_t* __restrict__ fslot) {
    const int p = blockIdx.x;
    const int f0 = pf[p], nf = pf[p + 1] - f0, a0 = pfa[p];
    for (int k = threadIdx.x; k < nf; k += blockDim.x) fslot[a0 + k] = slot_of[f0 + k];
}
// flag bits 3-6 = slot count (<= 15); chunk[c] = slots of nodes [32 c, 32 c + 32).
// The grid covers whole warps of 32 consecutive nodes.
__global__ void k_halo_flags(const int32_t* __restrict__ cnt, int64_t N, uint8_t* __restrict__ flags,
                             int32_t* __restrict__ chunk) {
    const int64_t N32 = (N + 31) / 32 * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N32; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = i < N ? cnt[i] : 0;
        if (i < N) flags[i] = (uint8_t)(flags[i] | (c << kHaloShift));
        const int sum = __reduce_add_sync(0xffffffffu, c);
        if ((threadIdx.x & 31) == 0) chunk[i / 32] = sum;
    }
}

// Largest number of a patch's elements that touch one patch-local node. One
// block per patch; counts in shared memory (max_local ints, by slot).
__global__ void k_patch_maxinc(const int32_t* __restrict__ pe, const int32_t* __restrict__ po,
                               const int32_t* __restrict__ pf, const uint32_t* __restrict__ lc, int32_t* maxinc) {
    extern __shared__ int cnt[];
    __shared__ int s_max;
    const int p = blockIdx.x;
    const int n_el = pe[p + 1] - pe[p];
    const int nloc = (po[p + 1] - po[p]) + (pf[p + 1] - pf[p]);
    const int nslot = nloc > 0 ? patch_slot(nloc - 1) + 1 : 0;  // lc holds slots
    for (int u = threadIdx.x; u < nslot; u += blockDim.x) cnt[u] = 0;
    if (threadIdx.x == 0) s_max = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < n_el * 10; t += blockDim.x) {
        const int j = t / 10, l = t % 10;
        const uint32_t w = lc[((int64_t)p * 5 + l / 2) * kPatchElems + j];
        const int u = (int)((l & 1) ? (w >> 16) : (w & 0xffffu));
        if (u < nslot) atomicAdd(&cnt[u], 1);
    }
    __syncthreads();
    int m = 0;
    for (int u = threadIdx.x; u < nslot; u += blockDim.x) m = max(m, cnt[u]);
    atomicMax(&s_max, m);
    __syncthreads();
    if (threadIdx.x == 0) maxinc[p] = s_max;
}

// max_e ||K_e||_inf per patch (row abs sums of K_e applied to the unit vectors,
// FP64 qdata), stored as double bits: non-negative doubles order like their bits.
template <class K>
__global__ void k_patch_knorm(const double* __restrict__ qd64, int64_t E, double cl, double cm,
                              unsigned long long* __restrict__ knorm) {
    constexpr int ND = 10 * K::DPN;
    const int64_t ne = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (ne >= E) return;
    const double* qd = qd64 + (ne / kPatchElems) * K::NQD * kPatchElems + ne % kPatchElems;
    double rs[ND];
#pragma unroll
    for (int i = 0; i < ND; ++i) rs[i] = 0.0;
    for (int j = 0; j < ND; ++j) {
        double x[ND], y[ND];
#pragma unroll
        for (int i = 0; i < ND; ++i) x[i] = i == j ? 1.0 : 0.0;
        K::apply(qd, kPatchElems, cl, cm, x, y);
#pragma unroll
        for (int i = 0; i < ND; ++i) rs[i] += fabs(y[i]);
    }
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) m = fmax(m, rs[i]);
    atomicMax(&knorm[ne / kPatchElems], (unsigned long long)__double_as_longlong(m));
}

// bound32[p] = maxinc[p] * max_e ||K_e||_inf * 1.001 (margin for the FP32 qdata and
// the rounding of the contributions), rounded up to FP32.
__global__ void k_patch_bound(const int32_t* __restrict__ maxinc, const unsigned long long* __restrict__ knorm,
                              int P, float* __restrict__ b32) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    b32[p] = __double2float_ru((double)maxinc[p] * __longlong_as_double((long long)knorm[p]) * 1.001);
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

// max_i |v_i w_i| as the bit pattern of a non-negative double
__global__ void k_max_abs_scaled(const double* v, const double* w, int64_t n, unsigned long long* out) {
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(v[i] * w[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
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
    geo::CtxRef ref;  // released after every buffer below
    const geo_mesh* mesh = nullptr;
    int phys = 0, dpn = 1, nq = 1;
    int64_t N = 0, E = 0, ndof = 0;
    int n_patches = 0, max_local = 0;
    double nu = 0, cl = 0, cm = 0, cd = 1.0, coef_scalar = 1.0;
    geo::DevBuf<int32_t> eperm, nperm, pe, po, pf, foreign;
    geo::DevBuf<uint32_t> lc;
    geo::DevBuf<uint8_t> flags;
    geo::DevBuf<uint8_t> mask_orig;  // Dirichlet mask, original DOF numbering
    geo::DevBuf<double> coef, qd64, g_new, diag_new, dinv64, ediag, diag_orig;
    geo::DevBuf<float> qd32, dinv32;
    // foreign ids and flags in aligned per-patch segments (bulk-copied with the elements)
    geo::DevBuf<int32_t> pfa, fids;
    geo::DevBuf<uint8_t> fflags;
    int max_for = 0;
    int max_own = 0;  // largest own-node count of a patch
    // halo mode of the PCG: slot of every foreign entry (fids
    // segments), slots before each 32-node chunk, and the slot arrays
    geo::DevBuf<int32_t> fslot, hbase;
    geo::DevBuf<double> halo64;
    geo::DevBuf<float> halo32;
    int64_t n_app = 0;
    bool halo_ok = false;  // slots built (every node has at most 15)
    int halo[2] = {0, 0};  // halo mode in use (FP64, FP32), see setup
    // per-patch bound of the fixed-point scatter (Scatter in mf_kernels.cuh)
    geo::DevBuf<int32_t> pmaxinc;
    geo::DevBuf<float> pbound32;
    geo::DevBuf<geo::PatchMeta> prec;  // per-patch records (PatchView::rec)
    // solver workspace
    geo::DevBuf<double> w64;
    geo::DevBuf<float> w32;
    geo::DevBuf<double> bvec, xvec;  // right-hand side and solution (patch numbering)
    // grow-only temporaries of the API calls (no cudaMalloc / cudaFree per call once
    // grown: cudaFree synchronises the device and can stall the caller)
    geo::DevBuf<double> tmp[7];
    geo::DevBuf<float> tmp32[2];
    geo::DevBuf<unsigned long long> tmpu[2];
    geo::DevBuf<geo::PcgState> state;
    geo::DevBuf<double> part;
    geo::PcgState* h_state = nullptr;  // pinned mirror
    int patch_grid[2] = {0, 0};        // resident patch-kernel blocks (FP64, FP32)
    int nbuf[2] = {2, 2};              // element-data buffers of the patch kernel (FP64, FP32)
    int own_bulk[2] = {0, 0};          // own-node slices by bulk copy (FP32 thermal PCG), see setup
    size_t patch_smem[2] = {0, 0};     // dynamic shared memory of the patch kernel
    int node_grid[2] = {0, 0};  // resident node-kernel blocks (FP64, mixed)
    // CUDA graphs of PCG iteration chunks, keyed by precision
    cudaGraphExec_t chunk[2] = {nullptr, nullptr};
    const void* chunk_key[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    ~geo_op() {
        for (auto& g : chunk)
            if (g) cudaGraphExecDestroy(g);
        if (h_state) cudaFreeHost(h_state);
    }
};

namespace geo {
namespace {

constexpr int kChunk = 16;  // PCG iterations per graph launch

inline unsigned nblk(int64_t n, int bs = 256) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, bs), 148 * 64));
}

template <class T>
T* grow(DevBuf<T>& b, size_t n) {
    b.ensure(n);
    return b.p;
}

PatchView view(const geo_op* op) {
    PatchView v;
    v.E = op->E;
    v.N = op->N;
    v.n_patches = op->n_patches;
    v.max_local = op->max_local;
    v.dpn = op->dpn;
    v.pe = op->pe.p;
    v.po = op->po.p;
    v.pf = op->pf.p;
    v.foreign = op->foreign.p;
    v.lc = op->lc.p;
    v.flags = op->flags.p;
    v.bound32 = op->pbound32.p;
    v.pfa = op->pfa.p;
    v.fids = op->fids.p;
    v.fflags = op->fflags.p;
    v.max_for = op->max_for;
    v.max_own = op->max_own;
    v.own_bulk = 0;
    v.fslot = op->fslot.p;
    v.halo = 0;
    v.rec = op->prec.p;
    return v;
}

// dynamic shared memory of the patch kernel: barriers, element-data buffers, node tables
template <class K, class T>
size_t smem_bytes(const geo_op* op, int nbuf, bool own, int halo = 0) {
    // xs (T), fixed-point accumulators (Scatter<T>::kWords INT32 words), flags (two
    // tables in the late loop shape), and for PCG the own-node slices
    const size_t flag_tables = nbuf == 2 ? patch_flag_tables<K, T, 2>() : patch_flag_tables<K, T, 1>();
    const size_t tables = (size_t)op->max_local * K::DPN * (sizeof(T) + 4 * Scatter<T>::kWords) +
                          (size_t)op->max_local * flag_tables + 16 +
                          (own ? (size_t)own_bytes<T>(op->max_own, K::DPN) : 0);
    return (nbuf == 2 ? patch_smem_tables<K, T, 2>(op->max_for, halo) : patch_smem_tables<K, T, 1>(op->max_for, halo)) +
           tables;
}

constexpr size_t kSmemLimit = 227 * 1024;

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

template <class K, class T, int NBUF>
int setup_patch_nbuf(size_t attr_bytes, size_t plain, size_t own, int& per_sm_plain) {
    GEO_CUDA(cudaFuncSetAttribute(k_patch<K, T, MODE_FREE, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)attr_bytes));
    GEO_CUDA(cudaFuncSetAttribute(k_patch<K, T, MODE_LIFT, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)attr_bytes));
    GEO_CUDA(cudaFuncSetAttribute(k_patch<K, T, MODE_PCG, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)attr_bytes));
    GEO_CUDA(cudaFuncSetAttribute(k_patch<K, T, MODE_PCG, NBUF, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)attr_bytes));
    GEO_CUDA(cudaFuncSetAttribute(k_patch<K, T, MODE_FREE, NBUF, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)attr_bytes));
    GEO_CUDA(cudaFuncSetAttribute(k_patch<K, T, MODE_LIFT, NBUF, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)attr_bytes));
    per_sm_plain = 0;
    GEO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_plain, k_patch<K, T, MODE_PCG, NBUF>, kPatchBS,
                                                           plain));
    int per_sm_own = 0;
    if (own)
        GEO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_own, k_patch<K, T, MODE_PCG, NBUF>,
                                                               kPatchBS, own));
    return per_sm_own;
}

// Picks double buffering when it fits in shared memory, and the own-node bulk copies
// (FP32 thermal PCG) when they cost no resident block: the gather then reads the
// patch's own-node D^-1, r and p_old from shared memory, but their buffer (about 13
// bytes per own node) took one block per SM away on meshes whose patches hold more
// nodes, which was slower than the plain gather (80^3, 112^3). Returns the grid.
template <class K, class T>
int setup_patch_kernels(geo_op* op, int slot) {
    int nbuf = 2;
    // GEO_PATCH_NBUF=1 forces the single-buffer kernel, so that tests cover it on small meshes
    const char* force_nbuf = std::getenv("GEO_PATCH_NBUF");
    if (smem_bytes<K, T>(op, 2, false) > kSmemLimit || (force_nbuf && std::strcmp(force_nbuf, "1") == 0)) {
        if (smem_bytes<K, T>(op, 1, false) > kSmemLimit)
            fail(GEO_ERR_UNSUPPORTED, "patch tables exceed shared memory (too many nodes per patch)");
        nbuf = 1;
    }
    op->nbuf[slot] = nbuf;
    const size_t plain = smem_bytes<K, T>(op, nbuf, false);
    size_t own = own_bulk<K, T, MODE_PCG>() ? smem_bytes<K, T>(op, nbuf, true) : 0;
    if (own > kSmemLimit) own = 0;
    int per_sm = 0;
    const int per_sm_own = nbuf == 2 ? setup_patch_nbuf<K, T, 2>(std::max(plain, own), plain, own, per_sm)
                                     : setup_patch_nbuf<K, T, 1>(std::max(plain, own), plain, own, per_sm);
    op->own_bulk[slot] = own && per_sm_own >= per_sm;
    op->patch_smem[slot] = op->own_bulk[slot] ? own : plain;
    if (per_sm < 1) fail(GEO_ERR_UNSUPPORTED, "patch kernel does not fit on an SM");
    per_sm = std::max(per_sm, per_sm_own);
    // halo mode: slots in the bulk copy when that costs no
    // resident block, else read by the flush from global memory. GEO_PATCH_HALO
    // (0: atomics, 1: slots in shared memory, 2: slots from global) forces a mode,
    // so that tests cover all three on small meshes.
    op->halo[slot] = 0;
    const char* force = std::getenv("GEO_PATCH_HALO");
    const int forced = force && force[0] >= '0' && force[0] <= '2' && force[1] == 0 ? force[0] - '0' : -1;
    if ((K::DPN == 1 || K::DPN == 3) && op->halo_ok && forced != 0) {
        op->halo[slot] = 2;
        const size_t hs = smem_bytes<K, T>(op, nbuf, op->own_bulk[slot] != 0, 1);
        int per_sm_halo = 0;
        if (hs <= kSmemLimit) {  // raises the limit of every mode (all launch with patch_smem[slot])
            const size_t attr = std::max(hs, std::max(plain, own));
            if (nbuf == 2) setup_patch_nbuf<K, T, 2>(attr, hs, 0, per_sm_halo);
            else setup_patch_nbuf<K, T, 1>(attr, hs, 0, per_sm_halo);
        }
        if (per_sm_halo > 0 && (forced == 1 || (forced < 0 && per_sm_halo >= per_sm))) {
            op->halo[slot] = 1;
            op->patch_smem[slot] = hs;
            if (forced == 1) per_sm = per_sm_halo;
        }
        if (forced == 2) {
            op->halo[slot] = 2;
            op->patch_smem[slot] = op->own_bulk[slot] ? own : plain;
        }
    }
    return per_sm * op->ctx->sm_count;
}

template <class K, class T, int MODE>
void launch_patch(const geo_op* op, int slot, cudaStream_t s, const T* qd, const PatchArgs<T>& pa) {
    const unsigned g = (unsigned)std::min(op->patch_grid[slot], op->n_patches);
    PatchView v = view(op);
    v.own_bulk = op->own_bulk[slot];
    v.halo = pa.halo ? op->halo[slot] : 0;  // halo mode whenever the caller passes the slot array
    const size_t smem = op->patch_smem[slot];
    const bool hg = v.halo == 2;
    if (op->nbuf[slot] == 2) {
        if (hg) k_patch<K, T, MODE, 2, 1><<<g, kPatchBS, smem, s>>>(v, qd, (T)op->cl, (T)op->cm, pa);
        else k_patch<K, T, MODE, 2><<<g, kPatchBS, smem, s>>>(v, qd, (T)op->cl, (T)op->cm, pa);
    } else {
        if (hg) k_patch<K, T, MODE, 1, 1><<<g, kPatchBS, smem, s>>>(v, qd, (T)op->cl, (T)op->cm, pa);
        else k_patch<K, T, MODE, 1><<<g, kPatchBS, smem, s>>>(v, qd, (T)op->cl, (T)op->cm, pa);
    }
}

// Halo slots (see k_halo_count): fslot in the fids
// segments (seg_total entries), the slot counts in flag bits 3-6, hbase, and the
// FP64 / FP32 slot arrays. Leaves op->halo_ok false (atomics kept) when some node
// has more than 15 foreign entries.
void build_halo_slots(geo_op* op, int64_t seg_total) {
    geo_ctx* ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    const int64_t N = op->N, A = op->n_app;
    DevBuf<int32_t> cnt(N), keys(A), vals(A), vals2(A), slot_of(A), mx(1);
    GEO_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes(), s));
    k_halo_count<<<nblk(A), 256, 0, s>>>(op->foreign.p, A, cnt.p);
    check_launch(ctx, "k_halo_count");
    size_t b1 = 0, b2 = 0;
    int bits = 1;
    while (bits < 31 && (int64_t(1) << bits) < N) ++bits;
    GEO_CUDA(cub::DeviceReduce::Max(nullptr, b1, cnt.p, mx.p, N, s));
    GEO_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b2, op->foreign.p, keys.p, vals.p, vals2.p, A, 0, bits, s));
    DevBuf<unsigned char> tmp(std::max(b1, b2));
    GEO_CUDA(cub::DeviceReduce::Max(tmp.p, b1, cnt.p, mx.p, N, s));
    int hmax = 0;
    GEO_CUDA(cudaMemcpyAsync(&hmax, mx.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    sync(ctx, "halo counts");
    if (hmax > 15) return;
    k_iota<<<nblk(A), 256, 0, s>>>(A, vals.p);
    check_launch(ctx, "k_iota");
    GEO_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, b2, op->foreign.p, keys.p, vals.p, vals2.p, A, 0, bits, s));
    k_halo_slot_of<<<nblk(A), 256, 0, s>>>(vals2.p, A, slot_of.p);
    check_launch(ctx, "k_halo_slot_of");
    op->fslot.alloc(seg_total + kForeignAlign);
    GEO_CUDA(cudaMemsetAsync(op->fslot.p, 0, op->fslot.bytes(), s));
    k_patch_fslot<<<(unsigned)op->n_patches, 128, 0, s>>>(op->pf.p, op->pfa.p, slot_of.p, op->fslot.p);
    check_launch(ctx, "k_patch_fslot");
    const int64_t nch = (N + 31) / 32;
    DevBuf<int32_t> chunk(nch + 1);
    GEO_CUDA(cudaMemsetAsync(chunk.p, 0, chunk.bytes(), s));
    k_halo_flags<<<nblk(nch * 32), 256, 0, s>>>(cnt.p, N, op->flags.p, chunk.p);
    check_launch(ctx, "k_halo_flags");
    op->hbase.alloc(nch + 1);
    size_t b3 = 0;
    GEO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b3, chunk.p, op->hbase.p, nch + 1, s));
    tmp.ensure(b3);
    GEO_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, b3, chunk.p, op->hbase.p, nch + 1, s));
    int total = 0;
    GEO_CUDA(cudaMemcpyAsync(&total, op->hbase.p + nch, sizeof(int), cudaMemcpyDeviceToHost, s));
    sync(ctx, "halo slots");
    if (total != A) fail(GEO_ERR_CUDA, "halo slot count mismatch");
    op->halo64.alloc(A * op->dpn);
    op->halo32.alloc(A * op->dpn);
    // slots of Dirichlet entries are never written (the node update ignores them)
    GEO_CUDA(cudaMemsetAsync(op->halo64.p, 0, op->halo64.bytes(), s));
    GEO_CUDA(cudaMemsetAsync(op->halo32.p, 0, op->halo32.bytes(), s));
    op->halo_ok = true;
}

// Recomputes qdata, diagonal, char_diag and the Jacobi inverse from op->coef.
void refresh_coefficients(geo_op* op) {
    geo_ctx* ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    const geo_mesh* m = op->mesh;
    reset_dev_err(ctx);
    const int nqd = (op->phys == 0 ? 6 : 10) * op->nq;
    op->qd64.ensure((size_t)nqd * op->n_patches * kPatchElems);
    op->qd32.ensure((size_t)nqd * op->n_patches * kPatchElems);
    GEO_CUDA(cudaMemsetAsync(op->qd64.p, 0, op->qd64.bytes(), s));
    GEO_CUDA(cudaMemsetAsync(op->qd32.p, 0, op->qd32.bytes(), s));
    if (op->nq == 1)
        k_qdata<1><<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->eperm.p, op->N, op->E,
                                                    op->coef.p, op->qd64.p, op->qd32.p, ctx->dev_err.p);
    else
        k_qdata<4><<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->eperm.p, op->N,
                                                              op->E, op->coef.p, op->qd64.p, op->qd32.p,
                                                              ctx->dev_err.p);
    check_launch(ctx, "k_qdata");
    {
        unsigned long long* knorm = grow(op->tmpu[0], (size_t)op->n_patches);
        GEO_CUDA(cudaMemsetAsync(knorm, 0, (size_t)op->n_patches * sizeof(unsigned long long), s));
        with_kernels(op, [&](auto k64, auto) {
            k_patch_knorm<decltype(k64)><<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->qd64.p, op->E, op->cl,
                                                                                   op->cm, knorm);
        });
        check_launch(ctx, "k_patch_knorm");
        op->pbound32.ensure(op->n_patches);
        k_patch_bound<<<(unsigned)cdiv(op->n_patches, 256), 256, 0, s>>>(op->pmaxinc.p, knorm, op->n_patches,
                                                                         op->pbound32.p);
        check_launch(ctx, "k_patch_bound");
        op->prec.ensure(op->n_patches);
        k_patch_records<<<(unsigned)cdiv(op->n_patches, 256), 256, 0, s>>>(view(op), op->prec.p);
        check_launch(ctx, "k_patch_records");
        sync(ctx, "patch bounds");
    }
    op->ediag.ensure((size_t)op->E * 10 * op->dpn);
    k_ediag<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->N, op->E, op->coef.p,
                                                       op->cl, op->cm, op->ediag.p, ctx->dev_err.p);
    check_launch(ctx, "k_ediag");
    raise_dev_err(ctx, read_dev_err(ctx), "operator set-up");
    op->diag_orig.ensure(op->ndof);
    k_gather_diag<<<(unsigned)cdiv(op->ndof, 256), 256, 0, s>>>(m->inc_ptr.p, m->inc.p, op->ediag.p, op->N,
                                                                op->dpn, op->diag_orig.p);
    check_launch(ctx, "k_gather_diag");
    unsigned long long* mx = grow(op->tmpu[1], 1);
    GEO_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long), s));
    k_max_abs<<<nblk(op->ndof), 256, 0, s>>>(op->diag_orig.p, op->ndof, mx);
    check_launch(ctx, "k_max_abs");
    unsigned long long bits = 0;
    GEO_CUDA(cudaMemcpyAsync(&bits, mx, sizeof(bits), cudaMemcpyDeviceToHost, s));
    sync(ctx, "char_diag");
    double maxd;
    std::memcpy(&maxd, &bits, sizeof(double));
    op->cd = maxd > 1.0 ? maxd : 1.0;  // assembly.rs:184-193
    // padded to whole 64-entry blocks: the patch kernel copies ranges rounded outwards to 16 bytes
    op->dinv64.ensure((size_t)(op->ndof + 63) / 64 * 64);
    // padded to whole 64-entry blocks: the patch kernel copies ranges rounded outwards to 4 values
    op->dinv32.ensure((size_t)(op->ndof + 63) / 64 * 64);
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
    op->ref.set(ctx);
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
    build_patches(s, op->N, mesh->xyz.p, op->E, mesh->conn.p, L);
    op->n_patches = L.n_patches;
    op->max_local = L.max_local;
    op->eperm = std::move(L.eperm);
    op->nperm = std::move(L.nperm);
    op->pe = std::move(L.patch_elem);
    op->po = std::move(L.patch_own);
    op->pf = std::move(L.patch_foreign);
    op->foreign = std::move(L.foreign);
    op->lc = std::move(L.lc);
    op->mask_orig.alloc(op->ndof);
    GEO_CUDA(cudaMemcpyAsync(op->mask_orig.p, dofs->mask.p, op->ndof, cudaMemcpyDeviceToDevice, s));
    // padded to 16 bytes: the patch kernel copies flag ranges rounded outwards to 16
    op->flags.alloc((size_t)(op->N + 15) / 16 * 16);
    GEO_CUDA(cudaMemsetAsync(op->flags.p, 0, op->flags.bytes(), s));
    op->g_new.alloc(op->ndof);
    k_node_flags<<<nblk(op->N), 256, 0, s>>>(op->nperm.p, L.shared.p, dofs->mask.p, dofs->vals.p, dpn, op->N,
                                             op->flags.p, op->g_new.p);
    check_launch(ctx, "k_node_flags");
    sync(ctx, "operator layout");
    {
        const int P = op->n_patches;
        std::vector<int32_t> pf(P + 1), pfa(P + 1), po(P + 1);
        GEO_CUDA(cudaMemcpy(pf.data(), op->pf.p, (P + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
        GEO_CUDA(cudaMemcpy(po.data(), op->po.p, (P + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
        for (int p = 0; p < P; ++p) op->max_own = std::max(op->max_own, po[p + 1] - po[p]);
        int64_t acc = 0;
        for (int p = 0; p < P; ++p) {
            const int nfor = pf[p + 1] - pf[p];
            op->max_for = std::max(op->max_for, nfor);
            pfa[p] = (int32_t)acc;
            acc += (nfor + kForeignAlign - 1) / kForeignAlign * kForeignAlign;
        }
        if (acc > INT32_MAX) fail(GEO_ERR_UNSUPPORTED, "too many foreign patch nodes");
        pfa[P] = (int32_t)acc;
        op->pfa.alloc(P + 1);
        GEO_CUDA(cudaMemcpy(op->pfa.p, pfa.data(), (P + 1) * sizeof(int32_t), cudaMemcpyHostToDevice));
        op->fids.alloc(acc + kForeignAlign);
        op->fflags.alloc(acc + kForeignAlign);
        GEO_CUDA(cudaMemsetAsync(op->fids.p, 0, op->fids.bytes(), s));
        GEO_CUDA(cudaMemsetAsync(op->fflags.p, 0, op->fflags.bytes(), s));
        k_patch_foreign<<<(unsigned)P, 128, 0, s>>>(op->pf.p, op->pfa.p, op->foreign.p, op->flags.p, op->fids.p,
                                                  op->fflags.p);
        check_launch(ctx, "k_patch_foreign");
        sync(ctx, "foreign segments");
        op->n_app = pf[P];
        if ((dpn == 1 || dpn == 3) && op->n_app > 0) build_halo_slots(op.get(), acc);
    }
    // affine (straight-sided) elements use one metric per element
    DevBuf<int> aff(1);
    GEO_CUDA(cudaMemsetAsync(aff.p, 0, sizeof(int), s));
    k_affine_check<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(mesh->xyz.p, mesh->conn.p, op->N, op->E, aff.p);
    check_launch(ctx, "k_affine_check");
    int curved = 0;
    GEO_CUDA(cudaMemcpyAsync(&curved, aff.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    sync(ctx, "affine check");
    op->nq = curved ? 4 : 1;
    if (op->max_local > 12288) fail(GEO_ERR_UNSUPPORTED, "patch tables exceed shared memory (too many nodes per patch)");
    op->pmaxinc.alloc(op->n_patches);
    k_patch_maxinc<<<(unsigned)op->n_patches, 128, (size_t)op->max_local * sizeof(int), s>>>(
        op->pe.p, op->po.p, op->pf.p, op->lc.p, op->pmaxinc.p);
    check_launch(ctx, "k_patch_maxinc");
    set_coef(op.get(), coef_e, coef);
    refresh_coefficients(op.get());
    with_kernels(op.get(), [&](auto k64, auto k32) {
        using K64 = decltype(k64);
        using K32 = decltype(k32);
        op->patch_grid[0] = setup_patch_kernels<K64, double>(op.get(), 0);
        op->patch_grid[1] = setup_patch_kernels<K32, float>(op.get(), 1);
    });
    with_kernels(op.get(), [&](auto k64, auto k32) {
        int per_sm = 0;
        if (op->halo[0])
            GEO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_pcg_update_halo<double, decltype(k64)::DPN, false>, kNodeBS, 0));
        else
            GEO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_pcg_update<double, decltype(k64)::DPN, false>, kNodeBS, 0));
        op->node_grid[0] = std::max(1, per_sm) * ctx->sm_count;
        if (op->halo[1])
            GEO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_pcg_update_halo<float, decltype(k32)::DPN, true>, kNodeBS, 0));
        else
            GEO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_pcg_update<float, decltype(k32)::DPN, true>, kNodeBS, 0));
        op->node_grid[1] = std::max(1, per_sm) * ctx->sm_count;
    });
    op->bvec.alloc(op->ndof);
    op->xvec.alloc(op->ndof);
    op->state.alloc(1);
    op->part.alloc((size_t)2 * std::max({op->patch_grid[0], op->patch_grid[1], op->node_grid[0], op->node_grid[1]}));
    GEO_CUDA(cudaMemset(op->state.p, 0, sizeof(PcgState)));
    GEO_CUDA(cudaMallocHost(&op->h_state, sizeof(PcgState)));
    return op.release();
}

// y = K_bc x in patch numbering (device vectors of type T)
template <class T>
void apply_new(geo_op* op, const T* x, T* y, int mode) {
    geo_ctx* ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    GEO_CUDA(cudaMemsetAsync(y, 0, op->ndof * sizeof(T), s));
    constexpr bool dbl = std::is_same<T, double>::value;
    const bool halo = op->halo[dbl ? 0 : 1] != 0;
    reset_dev_err(ctx);
    with_kernels(op, [&](auto k64, auto k32) {
        using K = typename std::conditional<dbl, decltype(k64), decltype(k32)>::type;
        const T* qd = dbl ? (const T*)op->qd64.p : (const T*)op->qd32.p;
        PatchArgs<T> pa{};
        pa.x = x;
        pa.y = y;
        pa.err = ctx->dev_err.p;
        if (halo) pa.halo = dbl ? (T*)op->halo64.p : (T*)op->halo32.p;
        if (mode == MODE_FREE) launch_patch<K, T, MODE_FREE>(op, dbl ? 0 : 1, s, qd, pa);
        else launch_patch<K, T, MODE_LIFT>(op, dbl ? 0 : 1, s, qd, pa);
    });
    check_launch(ctx, "k_patch");
    if (halo) {  // foreign contributions in slot order (and the Dirichlet rows of FREE)
        const T* h = dbl ? (const T*)op->halo64.p : (const T*)op->halo32.p;
        k_halo_combine<T><<<nblk(op->N), kNodeBS, 0, s>>>(op->flags.p, op->hbase.p, h, op->dpn, op->N, op->cd, x,
                                                          y, mode == MODE_FREE);
        check_launch(ctx, "k_halo_combine");
    } else if (mode == MODE_FREE) {
        k_dir_rows<T><<<nblk(op->ndof), 256, 0, s>>>(op->flags.p, op->dpn, op->ndof, op->cd, x, y);
        check_launch(ctx, "k_dir_rows");
    }
    raise_dev_err(ctx, read_dev_err(ctx), "matrix-free apply");
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
    double* fn = grow(op->tmp[4], (size_t)op->ndof);
    double* kg = grow(op->tmp[5], (size_t)op->ndof);
    to_new(op, f_orig_dev, fn);
    apply_new<double>(op, op->g_new.p, kg, MODE_LIFT);
    k_lift_finish<<<nblk(op->ndof), 256, 0, s>>>(op->flags.p, op->dpn, op->ndof, op->cd, fn, op->g_new.p, kg,
                                                fbc_new);
    check_launch(op->ctx, "k_lift_finish");
    sync(op->ctx, "lift");
}

// The node update of the PCG loop: the halo-mode kernel when the patch kernel runs
// in halo mode.
template <class K, class T, bool MIXED>
void launch_update(const geo_op* op, cudaStream_t s, const NodeArgs<T>& na) {
    constexpr int slot = std::is_same<T, double>::value ? 0 : 1;
    const unsigned g = (unsigned)op->node_grid[slot];
    if (op->halo[slot]) k_pcg_update_halo<T, K::DPN, MIXED><<<g, kNodeBS, 0, s>>>(na);
    else k_pcg_update<T, K::DPN, MIXED><<<g, kNodeBS, 0, s>>>(na);
}

// Enqueues one PCG iteration (patch kernel in PCG mode + node update).
template <class K, class T, bool MIXED>
void enqueue_iteration(geo_op* op, cudaStream_t s, const PatchArgs<T>& pa, const NodeArgs<T>& na) {
    constexpr bool dbl = std::is_same<T, double>::value;
    const T* qd = dbl ? (const T*)op->qd64.p : (const T*)op->qd32.p;
    launch_patch<K, T, MODE_PCG>(op, dbl ? 0 : 1, s, qd, pa);
    launch_update<K, T, MIXED>(op, s, na);
}

// Kernel arguments of the PCG loop over the operator's workspace (FP64 mode: r, q,
// p0, p1 in w64; mixed: w64 plus xs, r, q, p0, p1 in w32), allocated on first use.
struct PcgLaunchArgs {
    NodeArgs<double> n64{};
    NodeArgs<float> n32{};
    PatchArgs<double> p64{};
    PatchArgs<float> p32{};
};

PcgLaunchArgs pcg_args(geo_op* op, bool mixed) {
    const int64_t n = op->ndof;
    // sub-arrays at a common stride of whole 256-byte blocks, so that all vectors of
    // the node update share 16-byte alignment
    const int64_t np = (n + 63) / 64 * 64;
    op->w64.ensure((size_t)(mixed ? 1 : 4) * np);
    if (mixed) op->w32.ensure((size_t)5 * np);
    PcgLaunchArgs a;
    NodeArgs<double>& n64 = a.n64;
    NodeArgs<float>& n32 = a.n32;
    PatchArgs<double>& p64 = a.p64;
    PatchArgs<float>& p32 = a.p32;
    n64.flags = n32.flags = op->flags.p;
    n64.n = n32.n = n;
    n64.dpn = n32.dpn = op->dpn;
    n64.st = n32.st = p64.st = p32.st = op->state.p;
    p64.err = p32.err = &op->state.p->err;
    n64.part = n32.part = op->part.p;
    p64.part = p32.part = op->part.p;  // patch and node kernels never overlap
    n64.b = n32.b = op->bvec.p;
    n64.x64 = n32.x64 = op->xvec.p;
    if (!mixed) {
        n64.x = op->xvec.p;
        n64.r = op->w64.p;
        n64.q = op->w64.p + np;
        n64.pbuf0 = op->w64.p + 2 * np;
        n64.pbuf1 = op->w64.p + 3 * np;
        n64.dinv = op->dinv64.p;
        p64.r = n64.r;
        p64.dinv = n64.dinv;
        p64.pbuf0 = n64.pbuf0;
        p64.pbuf1 = n64.pbuf1;
        p64.y = n64.q;
    } else {
        n32.w64 = op->w64.p;
        n32.x = op->w32.p;
        n32.r = op->w32.p + np;
        n32.q = op->w32.p + 2 * np;
        n32.pbuf0 = op->w32.p + 3 * np;
        n32.pbuf1 = op->w32.p + 4 * np;
        n32.dinv = op->dinv32.p;
        p32.r = n32.r;
        p32.dinv = n32.dinv;
        p32.pbuf0 = n32.pbuf0;
        p32.pbuf1 = n32.pbuf1;
        p32.y = n32.q;
        p32.xsol = n32.x;  // updated by the patch kernel (z-form of the mixed solver)
    }
    if (op->halo[0]) {
        n64.halo = p64.halo = op->halo64.p;
        n64.hbase = op->hbase.p;
        n32.halo64 = op->halo64.p;  // the mixed solver's FP64 refresh apply
        n32.hbase = op->hbase.p;
    }
    if (op->halo[1]) {
        n32.halo = p32.halo = op->halo32.p;
        n32.hbase = op->hbase.p;
    }
    auto al = [](const void* q) { return ((uintptr_t)q & 15u) == 0; };
    n64.vec = al(n64.x) && al(n64.r) && al(n64.q) && al(n64.dinv) && al(n64.pbuf0) && al(n64.pbuf1);
    n32.vec = al(n32.x) && al(n32.r) && al(n32.q) && al(n32.dinv) && al(n32.pbuf0) && al(n32.pbuf1);
    return a;
}

// Writes the initial PcgState and launches the start kernels (x = 0, r = b, ||b||).
void pcg_start(geo_op* op, bool mixed, const PcgState& init, const PcgLaunchArgs& a) {
    cudaStream_t s = op->ctx->stream;
    GEO_CUDA(cudaMemcpyAsync(op->state.p, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    const unsigned ng = (unsigned)op->node_grid[mixed ? 1 : 0];
    if (mixed) {
        k_mixed_init1<<<ng, kNodeBS, 0, s>>>(a.n32);
        k_mixed_init2<<<ng, kNodeBS, 0, s>>>(a.n32);
    } else {
        k_pcg_init<double><<<ng, kNodeBS, 0, s>>>(a.n64);
    }
    check_launch(op->ctx, "pcg init");
}

// Jacobi-PCG on K_bc; b_new / x_new in patch numbering (device). Iterations run
// in CUDA-graph chunks of kChunk (kernels turn into no-ops once the device state
// says done or refresh); the host looks at the state between chunks and runs the
// FP64 refresh of the mixed solver when it is requested.
int solve_new(geo_op* op, const geo_cg_opts& o, geo_solver_stats* st) {
    geo_ctx* ctx = op->ctx;
    double* x_new = op->xvec.p;
    cudaStream_t s = ctx->stream;
    GEO_CHECK_ARG(o.use_preconditioner, "the matrix-free solver is Jacobi-preconditioned only");
    const bool mixed = o.precision == GEO_PRECISION_MIXED;
    PcgState init{};
    init.tol = o.tolerance;
    init.abs_tol = o.abs_tolerance;
    init.delta = o.reliable_delta;
    init.cd = op->cd;
    init.max_it = o.max_iterations;
    const PcgLaunchArgs la = pcg_args(op, mixed);
    const NodeArgs<float>& n32 = la.n32;
    const PatchArgs<double>& p64 = la.p64;
    const PatchArgs<float>& p32 = la.p32;
    const NodeArgs<double>& n64 = la.n64;
    const unsigned ng = (unsigned)op->node_grid[mixed ? 1 : 0];
    GEO_CUDA(cudaEventRecord(ctx->ev0, s));
    pcg_start(op, mixed, init, la);
    // (re)build the chunk graph when the buffers it captured changed
    const int pi = mixed ? 1 : 0;
    const void* key0 = mixed ? (const void*)op->w32.p : (const void*)op->w64.p;
    const void* key1 = (const void*)x_new;
    if (!op->chunk[pi] || op->chunk_key[pi][0] != key0 || op->chunk_key[pi][1] != key1) {
        if (op->chunk[pi]) cudaGraphExecDestroy(op->chunk[pi]);
        op->chunk[pi] = nullptr;
        cudaGraph_t g;
        GEO_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        with_kernels(op, [&](auto k64, auto k32) {
            for (int i = 0; i < kChunk; ++i) {
                if (mixed) enqueue_iteration<decltype(k32), float, true>(op, s, p32, n32);
                else enqueue_iteration<decltype(k64), double, false>(op, s, p64, n64);
            }
        });
        GEO_CUDA(cudaStreamEndCapture(s, &g));
        GEO_CUDA(cudaGraphInstantiate(&op->chunk[pi], g, 0));
        cudaGraphDestroy(g);
        op->chunk_key[pi][0] = key0;
        op->chunk_key[pi][1] = key1;
    }
    long long launches = mixed ? 2 : 1;
    const long long max_rounds = o.max_iterations / 1 + 64;
    for (long long round = 0; round <= max_rounds; ++round) {
        GEO_CUDA(cudaGraphLaunch(op->chunk[pi], s));
        launches += 2 * kChunk;
        GEO_CUDA(cudaMemcpyAsync(op->h_state, op->state.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        sync(ctx, "PCG chunk");
        if (op->h_state->err) fail(GEO_ERR_TIMEOUT, "matrix-free PCG: a bounded device-side wait timed out");
        if (op->h_state->flags & ST_DONE) break;
        if (mixed && (op->h_state->flags & ST_REFRESH)) {
            PatchArgs<double> ra{};
            ra.x = x_new;
            ra.y = op->w64.p;
            ra.err = &op->state.p->err;
            if (op->halo[0]) ra.halo = op->halo64.p;  // fixed-order foreign sums: bit-reproducible refresh
            k_refresh_flush<<<ng, kNodeBS, 0, s>>>(n32);
            with_kernels(op, [&](auto k64, auto) {
                launch_patch<decltype(k64), double, MODE_FREE>(op, 0, s, op->qd64.p, ra);
            });
            if (op->halo[0]) k_refresh_residual_halo<<<ng, kNodeBS, 0, s>>>(n32);
            else k_refresh_residual<<<ng, kNodeBS, 0, s>>>(n32);
            k_refresh_rescale<<<ng, kNodeBS, 0, s>>>(n32);
            check_launch(ctx, "refresh");
            launches += 4;
            GEO_CUDA(cudaMemcpyAsync(op->h_state, op->state.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
            sync(ctx, "refresh");
            if (op->h_state->err) fail(GEO_ERR_TIMEOUT, "matrix-free PCG: a bounded device-side wait timed out");
            if (op->h_state->flags & ST_DONE) break;
        }
    }
    if (mixed && !(op->h_state->flags & ST_CONVERGED)) {
        k_refresh_flush<<<ng, kNodeBS, 0, s>>>(n32);  // keep the FP32 correction
        check_launch(ctx, "final flush");
        launches += 1;
    }
    GEO_CUDA(cudaEventRecord(ctx->ev1, s));
    sync(ctx, "matrix-free PCG");
    float ms = 0.f;
    GEO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    const PcgState& h = *op->h_state;
    PcgResult r{h.it, h.res, h.bnorm, (h.flags & ST_CONVERGED) ? 1 : 0, (h.flags & ST_BREAKDOWN) ? 1 : 0, h.nupd};
    const int status = r.converged ? GEO_OK : (r.breakdown ? GEO_ERR_BREAKDOWN : GEO_NOT_CONVERGED);
    fill_stats(st, r, ms * 1e-3, status);
    if (st) st->kernel_launches = launches;
    return status;
}

// Device time of the two kernels of one PCG iteration, launch by launch: `iters`
// iterations from x = 0, r = op->bvec, with the stopping, refresh and
// iteration-limit tests unable to fire (tolerances 0, delta 0, no limit), so every
// launch does the full work of an iteration of a real solve. Events are
// recorded on the context stream between the launches.
void time_iterations(geo_op* op, bool mixed, int iters, double* patch_ms, double* update_ms) {
    geo_ctx* ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    PcgState init{};
    init.cd = op->cd;
    init.max_it = 1LL << 60;
    const PcgLaunchArgs la = pcg_args(op, mixed);
    pcg_start(op, mixed, init, la);
    std::vector<cudaEvent_t> ev((size_t)2 * iters + 1, nullptr);
    struct Guard {
        std::vector<cudaEvent_t>& v;
        ~Guard() {
            for (auto e : v)
                if (e) cudaEventDestroy(e);
        }
    } guard{ev};
    for (auto& e : ev) GEO_CUDA(cudaEventCreate(&e));
    with_kernels(op, [&](auto k64, auto k32) {
        for (int i = 0; i < iters; ++i) {
            GEO_CUDA(cudaEventRecord(ev[2 * i], s));
            if (mixed) launch_patch<decltype(k32), float, MODE_PCG>(op, 1, s, op->qd32.p, la.p32);
            else launch_patch<decltype(k64), double, MODE_PCG>(op, 0, s, op->qd64.p, la.p64);
            GEO_CUDA(cudaEventRecord(ev[2 * i + 1], s));
            if (mixed) launch_update<decltype(k32), float, true>(op, s, la.n32);
            else launch_update<decltype(k64), double, false>(op, s, la.n64);
        }
    });
    GEO_CUDA(cudaEventRecord(ev[2 * iters], s));
    check_launch(ctx, "timed PCG iterations");
    sync(ctx, "timed PCG iterations");
    PcgState h{};
    GEO_CUDA(cudaMemcpy(&h, op->state.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.err) fail(GEO_ERR_TIMEOUT, "matrix-free PCG: a bounded device-side wait timed out");
    if (h.flags & ST_DONE) fail(GEO_ERR_BREAKDOWN, "timed PCG iterations stopped early (breakdown)");
    double tp = 0.0, tu = 0.0;
    for (int i = 0; i < iters; ++i) {
        float a = 0.f, b = 0.f;
        GEO_CUDA(cudaEventElapsedTime(&a, ev[2 * i], ev[2 * i + 1]));
        GEO_CUDA(cudaEventElapsedTime(&b, ev[2 * i + 1], ev[2 * i + 2]));
        tp += a;
        tu += b;
    }
    *patch_ms = tp / iters;
    *update_ms = tu / iters;
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
    const double* dx = stage_in(x, n, op->tmp[0], s);
    double* yo = grow(op->tmp[3], (size_t)n);
    if (precision == GEO_PRECISION_MIXED) {
        float* x32 = grow(op->tmp32[0], (size_t)n);
        float* y32 = grow(op->tmp32[1], (size_t)n);
        k_to_new<double, float><<<nblk(n), 256, 0, s>>>(op->nperm.p, op->dpn, op->N, dx, x32);
        apply_new<float>(op, x32, y32, MODE_FREE);
        k_to_orig<float, double><<<nblk(n), 256, 0, s>>>(op->nperm.p, op->dpn, op->N, y32, yo);
        check_launch(op->ctx, "k_to_orig");
        copy_out(y, yo, n, s);
        sync(op->ctx, "geo_op_apply");
    } else {
        double* xn = grow(op->tmp[1], (size_t)n);
        double* yn = grow(op->tmp[2], (size_t)n);
        to_new(op, dx, xn);
        apply_new<double>(op, xn, yn, MODE_FREE);
        to_orig(op, yn, yo);
        copy_out(y, yo, n, s);
        sync(op->ctx, "geo_op_apply");
    }
    GEO_API_END
}

int geo_op_lift_rhs(geo_op* op, const double* f, double* f_bc) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && f && f_bc, "NULL argument");
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    const double* df = stage_in(f, n, op->tmp[0], s);
    double* fb = grow(op->tmp[1], (size_t)n);
    double* fo = grow(op->tmp[2], (size_t)n);
    lift_new(op, df, fb);
    to_orig(op, fb, fo);
    copy_out(f_bc, fo, n, s);
    sync(op->ctx, "geo_op_lift_rhs");
    GEO_API_END
}

int geo_op_diagonal(geo_op* op, double* diag) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && diag, "NULL argument");
    double* d = grow(op->tmp[0], (size_t)op->ndof);
    to_orig(op, op->diag_new.p, d);
    copy_out(diag, d, op->ndof, op->ctx->stream);
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
    const double* db = stage_in(b, n, op->tmp[0], s);
    to_new(op, db, op->bvec.p);
    const int status = solve_new(op, o, st);
    double* dst = x;
    if (!is_device_ptr(x)) dst = grow(op->tmp[1], (size_t)n);
    to_orig(op, op->xvec.p, dst);
    if (dst != x) copy_out(x, dst, n, s);
    sync(op->ctx, "geo_cg_solve_matfree");
    return finish_status(op->ctx, status);
    GEO_API_END
}

int geo_op_element_gradient(geo_op* op, const double* u, const double* lambda, double* grad_e) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && u && lambda && grad_e, "NULL argument");
    cudaStream_t s = op->ctx->stream;
    const double* du = stage_in(u, op->ndof, op->tmp[0], s);
    const double* dl = stage_in(lambda, op->ndof, op->tmp[1], s);
    double* g = grow(op->tmp[6], (size_t)op->E);
    const geo_mesh* m = op->mesh;
    k_elem_gradient<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->N, op->E,
                                                               op->coef.p, op->cl, op->cm, op->mask_orig.p, du, dl,
                                                               g);
    check_launch(op->ctx, "k_elem_gradient");
    copy_out(grad_e, g, op->E, s);
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
    const double* df = stage_in(f, n, op->tmp[0], s);
    lift_new(op, df, op->bvec.p);
    const int status = solve_new(op, o, st);
    double* dst = u;
    if (!is_device_ptr(u)) dst = grow(op->tmp[1], (size_t)n);
    to_orig(op, op->xvec.p, dst);
    if (dst != u) copy_out(u, dst, n, s);
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
    double* lo = grow(op->tmp[3], (size_t)n);
    double* ge = grow(op->tmp[6], (size_t)op->E);
    const double* du = nullptr;
    if (u) {
        du = stage_in(u, n, op->tmp[0], s);
    } else {
        // recompute the forward solution instead of storing it
        const double* df = stage_in(f, n, op->tmp[0], s);
        lift_new(op, df, op->bvec.p);
        const int fs = solve_new(op, o, nullptr);
        if (fs != GEO_OK) return finish_status(op->ctx, fs);
        double* uo = grow(op->tmp[2], (size_t)n);
        to_orig(op, op->xvec.p, uo);
        du = uo;
    }
    // adjoint right-hand side: dJ/du on free DOFs, zero on Dirichlet DOFs (K_bc
    // is symmetric and its Dirichlet rows are decoupled, so lambda_D = 0)
    const double* dg = stage_in(dJ_du, n, op->tmp[1], s);
    to_new(op, dg, op->bvec.p);
    k_zero_dir<double><<<nblk(n), 256, 0, s>>>(op->flags.p, op->dpn, n, op->bvec.p);
    check_launch(op->ctx, "adjoint rhs");
    // The adjoint system is linear in its right-hand side: solve with dJ/du scaled
    // so that its Jacobi-preconditioned form D^-1 b has unit max-norm (lambda is
    // then O(1)) and scale lambda back, so that the absolute breakdown and
    // stopping thresholds of the CG loop do not depend on the misfit's units or
    // on the stiffness scale.
    unsigned long long* mx = grow(op->tmpu[1], 1);
    GEO_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long), s));
    k_max_abs_scaled<<<nblk(n), 256, 0, s>>>(op->bvec.p, op->dinv64.p, n, mx);
    unsigned long long bits = 0;
    GEO_CUDA(cudaMemcpyAsync(&bits, mx, sizeof(bits), cudaMemcpyDeviceToHost, s));
    sync(op->ctx, "adjoint scale");
    double zmax;
    std::memcpy(&zmax, &bits, sizeof(double));
    int status = GEO_OK;
    if (zmax > 0.0) {
        k_scale<<<nblk(n), 256, 0, s>>>(op->bvec.p, n, 1.0 / zmax);  // b / zmax
        status = solve_new(op, o, st);
        k_scale<<<nblk(n), 256, 0, s>>>(op->xvec.p, n, zmax);        // lambda = zmax * lambda_scaled
    } else {
        GEO_CUDA(cudaMemsetAsync(op->xvec.p, 0, n * sizeof(double), s));
    }
    to_orig(op, op->xvec.p, lo);
    const geo_mesh* m = op->mesh;
    k_elem_gradient<<<(unsigned)cdiv(op->E, 128), 128, 0, s>>>(op->phys, m->xyz.p, m->conn.p, op->N, op->E,
                                                               op->coef.p, op->cl, op->cm, op->mask_orig.p, du,
                                                               lo, ge);
    check_launch(op->ctx, "k_elem_gradient");
    copy_out(dJ_dlncoef, ge, op->E, s);
    sync(op->ctx, "geo_vjp");
    return finish_status(op->ctx, status);
    GEO_API_END
}

int geo_op_time_pcg_kernels(geo_op* op, const double* b, int32_t precision, int32_t iterations, double* patch_ms,
                            double* update_ms) {
    GEO_API_BEGIN(op ? op->ctx : nullptr)
    GEO_CHECK_ARG(op && b && patch_ms && update_ms, "NULL argument");
    GEO_CHECK_ARG(iterations >= 1 && iterations <= 4096, "iterations must be in [1, 4096]");
    cudaStream_t s = op->ctx->stream;
    const double* db = stage_in(b, op->ndof, op->tmp[0], s);
    to_new(op, db, op->bvec.p);
    time_iterations(op, precision == GEO_PRECISION_MIXED, iterations, patch_ms, update_ms);
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
