// K1: element integration (FP64), one thread per element row / 3x3 block.
//
// Follows the reference's isoparametric formulation: at every quadrature point
// the Jacobian is rebuilt from all 10 node coordinates (basis.rs:196-223), so
// curved Tet10 elements integrate exactly as in the reference.
#include <algorithm>

#include "objects.h"
#include "tet10.cuh"

namespace geo {

__device__ __forceinline__ void load_nodes(const double* __restrict__ xyz, const int32_t* __restrict__ conn,
                                           int64_t N, int64_t E, int64_t e, double (&X)[10][3]) {
#pragma unroll
    for (int l = 0; l < 10; ++l) {
        const int64_t n = conn[l * E + e];
        X[l][0] = xyz[n];
        X[l][1] = xyz[N + n];
        X[l][2] = xyz[2 * N + n];
    }
}

// Geometry at 4-point QP q: Jinv and w*|det| (element.rs:36-40). Returns false
// when det == 0 (basis.rs:247).
__device__ __forceinline__ bool qp_geometry(const double (&X)[10][3], int q, double (&Ji)[3][3],
                                            double& wdet) {
    double L[4], J[3][3], A[3][3];
    qp4(q, L);
    jacobian10(X, L, J);
    const double d = det3(J);
    if (d == 0.0) return false;
    adj3(J, A);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) Ji[r][c] = A[r][c] / d;
    wdet = kQw * fabs(d);
    return true;
}

// ElementMatrix::thermal_stiffness (element.rs:23-61); thread (e, i) -> row i.
__global__ void k_thermal_stiffness(const double* __restrict__ xyz, const int32_t* __restrict__ conn,
                                    int64_t N, int64_t E, const double* __restrict__ k_e, double k,
                                    double* __restrict__ out, int* err) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= E * 10) return;
    const int64_t e = t / 10;
    const int i = (int)(t % 10);
    double X[10][3];
    load_nodes(xyz, conn, N, E, e, X);
    const double kk = k_e ? k_e[e] : k;
    double row[10];
#pragma unroll
    for (int j = 0; j < 10; ++j) row[j] = 0.0;
    for (int q = 0; q < 4; ++q) {
        double Ji[3][3], w;
        if (!qp_geometry(X, q, Ji, w)) {
            atomicOr(err, DEV_ERR_SINGULAR);
            return;
        }
        double L[4], g[3], gi[3];
        qp4(q, L);
        ref_grad(i, L, g);
        cart_grad(Ji, g, gi);
#pragma unroll
        for (int j = 0; j < 10; ++j) {
            double gj[3];
            ref_grad(j, L, g);
            cart_grad(Ji, g, gj);
            const double gd = gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2];
            row[j] += kk * gd * w;
        }
    }
    double* o = out + e * 100 + i * 10;
#pragma unroll
    for (int j = 0; j < 10; ++j) o[j] = row[j];
}

// ElementMatrix::thermal_mass (element.rs:74-105), 5-point rule.
__global__ void k_thermal_mass(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N,
                               int64_t E, double rho_cp, double* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= E * 10) return;
    const int64_t e = t / 10;
    const int i = (int)(t % 10);
    double X[10][3];
    load_nodes(xyz, conn, N, E, e, X);
    double row[10];
#pragma unroll
    for (int j = 0; j < 10; ++j) row[j] = 0.0;
    for (int q = 0; q < 5; ++q) {
        double L[4], J[3][3], Nf[10];
        qp5(q, L);
        jacobian10(X, L, J);
        const double w = qw5(q) * fabs(det3(J));
        shape_n(L, Nf);
#pragma unroll
        for (int j = 0; j < 10; ++j) row[j] += rho_cp * Nf[i] * Nf[j] * w;
    }
    double* o = out + e * 100 + i * 10;
#pragma unroll
    for (int j = 0; j < 10; ++j) o[j] = row[j];
}

// ElementMatrix::thermal_load (element.rs:117-140); thread per element.
__global__ void k_thermal_load(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N,
                               int64_t E, double Q, double* __restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    double X[10][3];
    load_nodes(xyz, conn, N, E, e, X);
    double f[10];
#pragma unroll
    for (int i = 0; i < 10; ++i) f[i] = 0.0;
    for (int q = 0; q < 4; ++q) {
        double L[4], J[3][3], Nf[10];
        qp4(q, L);
        jacobian10(X, L, J);
        const double w = kQw * fabs(det3(J));
        shape_n(L, Nf);
#pragma unroll
        for (int i = 0; i < 10; ++i) f[i] += Nf[i] * Q * w;
    }
#pragma unroll
    for (int i = 0; i < 10; ++i) out[e * 10 + i] = f[i];
}

// ElasticityElement::stiffness_matrix (mechanics/element.rs:33-65) with the
// isotropic D of constitutive.rs:63-102; thread (e, i, j) -> 3x3 block (i, j).
// B^T D B for isotropic D expands to
//   K^{ij}_{ab} = sum_q w|detJ| (lam g_ia g_jb + mu (g_ib g_ja + delta_ab g_i.g_j)).
__global__ void k_elasticity_stiffness(const double* __restrict__ xyz, const int32_t* __restrict__ conn,
                                       int64_t N, int64_t E, const double* __restrict__ E_e, double Ey,
                                       double nu, double* __restrict__ out, int* err) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= E * 100) return;
    const int64_t e = t / 100;
    const int i = (int)((t % 100) / 10), j = (int)(t % 10);
    double X[10][3];
    load_nodes(xyz, conn, N, E, e, X);
    const double Ev = E_e ? E_e[e] : Ey;
    const double factor = Ev / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double lam = factor * nu;
    const double mu = factor * ((1.0 - 2.0 * nu) / 2.0);
    double K[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < 4; ++q) {
        double Ji[3][3], w;
        if (!qp_geometry(X, q, Ji, w)) {
            atomicOr(err, DEV_ERR_SINGULAR);
            return;
        }
        double L[4], g[3], gi[3], gj[3];
        qp4(q, L);
        ref_grad(i, L, g);
        cart_grad(Ji, g, gi);
        ref_grad(j, L, g);
        cart_grad(Ji, g, gj);
        const double dd = gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
                K[a][b] += w * (lam * gi[a] * gj[b] + mu * (gi[b] * gj[a] + (a == b ? dd : 0.0)));
    }
    double* o = out + e * 900;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) o[(3 * i + a) * 30 + 3 * j + b] = K[a][b];
}

// BodyForce::gravity_load (mechanics/body_force.rs:49-84); thread per element.
__global__ void k_gravity_load(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N,
                               int64_t E, double rho, double gx, double gy, double gz,
                               double* __restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    double X[10][3];
    load_nodes(xyz, conn, N, E, e, X);
    const double bf[3] = {rho * gx, rho * gy, rho * gz};
    double f[30];
#pragma unroll
    for (int i = 0; i < 30; ++i) f[i] = 0.0;
    for (int q = 0; q < 4; ++q) {
        double L[4], J[3][3], Nf[10];
        qp4(q, L);
        jacobian10(X, L, J);
        const double w = kQw * fabs(det3(J));
        shape_n(L, Nf);
#pragma unroll
        for (int i = 0; i < 10; ++i)
#pragma unroll
            for (int a = 0; a < 3; ++a) f[3 * i + a] += w * Nf[i] * bf[a];
    }
#pragma unroll
    for (int i = 0; i < 30; ++i) out[e * 30 + i] = f[i];
}

inline unsigned grid_for(int64_t n, int bs) { return (unsigned)cdiv(n, bs); }

// Internal launchers (used by the assemblers); outputs are device buffers.
void element_thermal_stiffness(geo_ctx* ctx, const geo_mesh* m, const double* k_e_dev, double k,
                               double* out) {
    k_thermal_stiffness<<<grid_for(m->n_elem * 10, 128), 128, 0, ctx->stream>>>(
        m->xyz.p, m->conn.p, m->n_nodes, m->n_elem, k_e_dev, k, out, ctx->dev_err.p);
    check_launch(ctx, "k_thermal_stiffness");
}

void element_thermal_load(geo_ctx* ctx, const geo_mesh* m, double Q, double* out) {
    k_thermal_load<<<grid_for(m->n_elem, 128), 128, 0, ctx->stream>>>(m->xyz.p, m->conn.p, m->n_nodes,
                                                                       m->n_elem, Q, out);
    check_launch(ctx, "k_thermal_load");
}

void element_elasticity_stiffness(geo_ctx* ctx, const geo_mesh* m, const double* E_dev, double E,
                                  double nu, double* out) {
    k_elasticity_stiffness<<<grid_for(m->n_elem * 100, 128), 128, 0, ctx->stream>>>(
        m->xyz.p, m->conn.p, m->n_nodes, m->n_elem, E_dev, E, nu, out, ctx->dev_err.p);
    check_launch(ctx, "k_elasticity_stiffness");
}

void element_gravity_load(geo_ctx* ctx, const geo_mesh* m, double rho, const double g[3], double* out) {
    k_gravity_load<<<grid_for(m->n_elem, 128), 128, 0, ctx->stream>>>(m->xyz.p, m->conn.p, m->n_nodes,
                                                                       m->n_elem, rho, g[0], g[1], g[2], out);
    check_launch(ctx, "k_gravity_load");
}

}  // namespace geo

using namespace geo;

namespace {

// Runs `launch(dev_out)` and delivers n doubles to the caller's out pointer.
template <class F>
void run_to(geo_ctx* ctx, double* out, size_t n, F&& launch) {
    DevBuf<double> tmp;
    double* dst = out;
    const bool dev = is_device_ptr(out);
    if (!dev) {
        tmp.alloc(n);
        dst = tmp.p;
    }
    reset_dev_err(ctx);
    launch(dst);
    if (!dev) copy_out(out, dst, n, ctx->stream);
    const int bits = read_dev_err(ctx);
    raise_dev_err(ctx, bits, "element integration");
}

}  // namespace

extern "C" {

int geo_element_thermal_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const double* k_e, double k,
                                  double* ke) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && ke, "NULL argument");
    DevBuf<double> tk;
    const double* dk = k_e ? stage_in(k_e, mesh->n_elem, tk, ctx->stream) : nullptr;
    run_to(ctx, ke, mesh->n_elem * 100, [&](double* o) { element_thermal_stiffness(ctx, mesh, dk, k, o); });
    GEO_API_END
}

int geo_element_thermal_mass(geo_ctx* ctx, const geo_mesh* mesh, double density, double specific_heat,
                             double* me) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && me, "NULL argument");
    run_to(ctx, me, mesh->n_elem * 100, [&](double* o) {
        k_thermal_mass<<<grid_for(mesh->n_elem * 10, 128), 128, 0, ctx->stream>>>(
            mesh->xyz.p, mesh->conn.p, mesh->n_nodes, mesh->n_elem, density * specific_heat, o);
        check_launch(ctx, "k_thermal_mass");
    });
    GEO_API_END
}

int geo_element_thermal_load(geo_ctx* ctx, const geo_mesh* mesh, double source, double* fe) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && fe, "NULL argument");
    run_to(ctx, fe, mesh->n_elem * 10, [&](double* o) { element_thermal_load(ctx, mesh, source, o); });
    GEO_API_END
}

int geo_element_elasticity_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const double* E_e, double E,
                                     double nu, double* ke) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && ke, "NULL argument");
    GEO_CHECK_ARG(nu > -1.0 && nu < 0.5, "Poisson's ratio must be in (-1, 0.5)");
    DevBuf<double> tE;
    const double* dE = E_e ? stage_in(E_e, mesh->n_elem, tE, ctx->stream) : nullptr;
    run_to(ctx, ke, mesh->n_elem * 900,
           [&](double* o) { element_elasticity_stiffness(ctx, mesh, dE, E, nu, o); });
    GEO_API_END
}

int geo_element_gravity_load(geo_ctx* ctx, const geo_mesh* mesh, double density, const double gravity[3],
                             double* fe) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && fe && gravity, "NULL argument");
    run_to(ctx, fe, mesh->n_elem * 30, [&](double* o) { element_gravity_load(ctx, mesh, density, gravity, o); });
    GEO_API_END
}

}  // extern "C"
