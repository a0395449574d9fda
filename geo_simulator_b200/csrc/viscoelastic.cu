// Maxwell viscoelasticity: the history force of
// Assembler::assemble_maxwell_viscoelastic_parallel (fem/assembly.rs:959-1020,
// element part ElasticityElement::maxwell_viscoelastic, mechanics/element.rs:257-296)
// and update_stresses_maxwell (mechanics/stress_update.rs:39-143).
//
// One thread per element evaluates the isoparametric B at the 4 points in FP64.
// The history force f_e = -sum_q w_q |det J_q| B_q^T sigma_n is gathered per node
// through the node -> (element, local node) inverse map in element order, so the
// sums are deterministic; the stiffness is the elastic one (the reference
// assembles the elastic D and leaves the relaxation to the stress update).
#include <cmath>

#include "objects.h"
#include "tet10.cuh"

namespace geo {
namespace {

inline unsigned nb(int64_t n, int bs = 128) { return (unsigned)std::max<int64_t>(1, cdiv(n, bs)); }

__device__ __forceinline__ void elem_coords(const double* __restrict__ xyz, const int32_t* __restrict__ conn,
                                            int64_t N, int64_t E, int64_t e, int32_t (&nd)[10],
                                            double (&X)[10][3]) {
#pragma unroll
    for (int l = 0; l < 10; ++l) {
        nd[l] = conn[l * E + e];
        X[l][0] = xyz[nd[l]];
        X[l][1] = xyz[N + nd[l]];
        X[l][2] = xyz[2 * N + nd[l]];
    }
}

// Cartesian shape-function gradients dN[10][3] at 4-point quadrature point q and
// w |det J|; false on a singular Jacobian.
__device__ __forceinline__ bool qp_gradients(const double (&X)[10][3], int q, double (&dN)[10][3], double& wdet) {
    double L[4], J[3][3], A[3][3];
    qp4(q, L);
    jacobian10(X, L, J);
    const double d = det3(J);
    if (d == 0.0) return false;
    adj3(J, A);
    double Ji[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) Ji[r][c] = A[r][c] / d;
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        double g[3];
        ref_grad(i, L, g);
        cart_grad(Ji, g, dN[i]);
    }
    wdet = kQw * fabs(d);
    return true;
}

// fe[e][3 i + c] = -sum_q w |det J| (B^T sigma)_(3 i + c); B rows [xx yy zz xy yz zx]
// with engineering shears (mechanics/strain.rs:38-71).
__global__ void k_maxwell_force(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N,
                                int64_t E, const double* __restrict__ stress, double* __restrict__ fe, int* err) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    int32_t nd[10];
    double X[10][3];
    elem_coords(xyz, conn, N, E, e, nd, X);
    double s[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = stress[6 * e + k];
    double f[30];
#pragma unroll
    for (int i = 0; i < 30; ++i) f[i] = 0.0;
    for (int q = 0; q < 4; ++q) {
        double dN[10][3], w;
        if (!qp_gradients(X, q, dN, w)) {
            atomicOr(err, DEV_ERR_SINGULAR);
            return;
        }
#pragma unroll
        for (int i = 0; i < 10; ++i) {
            const double dx = dN[i][0], dy = dN[i][1], dz = dN[i][2];
            f[3 * i + 0] -= w * (dx * s[0] + dy * s[3] + dz * s[5]);
            f[3 * i + 1] -= w * (dy * s[1] + dx * s[3] + dz * s[4]);
            f[3 * i + 2] -= w * (dz * s[2] + dy * s[4] + dx * s[5]);
        }
    }
#pragma unroll
    for (int i = 0; i < 30; ++i) fe[30 * e + i] = f[i];
}

// f[3 i + c] = sum over the incidences of node i (element order) of fe
__global__ void k_gather3(const int32_t* __restrict__ ptr, const int32_t* __restrict__ inc,
                          const double* __restrict__ fe, int64_t N, double* __restrict__ f) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int64_t i = t / 3;
    const int c = (int)(t % 3);
    double s = 0.0;
    for (int32_t p = ptr[i]; p < ptr[i + 1]; ++p) {
        const int32_t el = inc[p];
        s = __dadd_rn(s, fe[(int64_t)(el / 10) * 30 + 3 * (el % 10) + c]);
    }
    f[t] = s;
}

// sigma_{n+1}: strain increment averaged over the 4 points, elastic predictor,
// deviatoric part scaled by `factor` = 1 / (1 + dt / tau_M)
__global__ void k_maxwell_update(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N,
                                 int64_t E, double G, double lam, double factor, const double* __restrict__ u_n,
                                 const double* __restrict__ u_next, const double* __restrict__ s_n,
                                 double* __restrict__ s_next, int* err) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    int32_t nd[10];
    double X[10][3];
    elem_coords(xyz, conn, N, E, e, nd, X);
    double du[10][3];
#pragma unroll
    for (int i = 0; i < 10; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) du[i][c] = u_next[3 * (int64_t)nd[i] + c] - u_n[3 * (int64_t)nd[i] + c];
    double de[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < 4; ++q) {
        double dN[10][3], w;
        if (!qp_gradients(X, q, dN, w)) {
            atomicOr(err, DEV_ERR_SINGULAR);
            return;
        }
        double b[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int i = 0; i < 10; ++i) {
            const double dx = dN[i][0], dy = dN[i][1], dz = dN[i][2];
            b[0] += dx * du[i][0];
            b[1] += dy * du[i][1];
            b[2] += dz * du[i][2];
            b[3] += dy * du[i][0] + dx * du[i][1];
            b[4] += dz * du[i][1] + dy * du[i][2];
            b[5] += dx * du[i][2] + dz * du[i][0];
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) de[k] += b[k];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) de[k] /= 4.0;
    const double* sn = s_n + 6 * e;
    const double tr = de[0] + de[1] + de[2];
    const double st0 = sn[0] + lam * tr + 2.0 * G * de[0];
    const double st1 = sn[1] + lam * tr + 2.0 * G * de[1];
    const double st2 = sn[2] + lam * tr + 2.0 * G * de[2];
    const double p = (st0 + st1 + st2) / 3.0;
    double* o = s_next + 6 * e;
    o[0] = (st0 - p) * factor + p;
    o[1] = (st1 - p) * factor + p;
    o[2] = (st2 - p) * factor + p;
    o[3] = (sn[3] + G * de[3]) * factor;
    o[4] = (sn[4] + G * de[4]) * factor;
    o[5] = (sn[5] + G * de[5]) * factor;
}

void check_material(double E, double nu, double mu) {
    GEO_CHECK_ARG(E > 0.0, "Young's modulus must be positive");
    GEO_CHECK_ARG(nu > -1.0 && nu < 0.5, "Poisson's ratio must be in (-1, 0.5)");
    GEO_CHECK_ARG(mu > 0.0, "Viscosity must be positive");
}

void history_force(geo_ctx* ctx, geo_mesh* m, const double* stress, double* f_dev) {
    cudaStream_t s = ctx->stream;
    ensure_inverse_map(m);
    double* fe = ctx_scratch<double>(ctx, SCR_TMP0, (size_t)(30 * m->n_elem));
    const double* ds = stage_in(ctx, SCR_IN0, stress, (size_t)(6 * m->n_elem));
    reset_dev_err(ctx);
    k_maxwell_force<<<nb(m->n_elem), 128, 0, s>>>(m->xyz.p, m->conn.p, m->n_nodes, m->n_elem, ds, fe,
                                                  ctx->dev_err.p);
    check_launch(ctx, "k_maxwell_force");
    raise_dev_err(ctx, read_dev_err(ctx), "maxwell history force");
    k_gather3<<<nb(3 * m->n_nodes, 256), 256, 0, s>>>(m->inc_ptr.p, m->inc.p, fe, m->n_nodes, f_dev);
    check_launch(ctx, "k_gather3");
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

int geo_maxwell_history_force(geo_ctx* ctx, const geo_mesh* mesh, const double* stress, double* f) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && stress && f, "NULL argument");
    geo_mesh* m = const_cast<geo_mesh*>(mesh);
    double* out = ctx_scratch<double>(ctx, SCR_OUT0, (size_t)(3 * m->n_nodes));
    history_force(ctx, m, stress, out);
    copy_out(f, out, (size_t)(3 * m->n_nodes), ctx->stream);
    sync(ctx, "geo_maxwell_history_force");
    GEO_API_END
}

int geo_assemble_maxwell_viscoelastic(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, double E, double nu,
                                      double mu, double dt, const double* stress, geo_csr** K, double* f_history) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && dofs && stress && K && f_history, "NULL argument");
    GEO_CHECK_ARG(dofs->dpn == 3, "Maxwell viscoelasticity requires 3 DOF per node");
    check_material(E, nu, mu);
    (void)dt;  // the reference assembles the elastic stiffness for every dt
    const int rc = geo_assemble_elasticity_stiffness(ctx, mesh, dofs, nullptr, E, nu, K);
    if (rc != GEO_OK) return rc;
    geo_mesh* m = const_cast<geo_mesh*>(mesh);
    double* out = ctx_scratch<double>(ctx, SCR_OUT0, (size_t)(3 * m->n_nodes));
    history_force(ctx, m, stress, out);
    copy_out(f_history, out, (size_t)(3 * m->n_nodes), ctx->stream);
    sync(ctx, "geo_assemble_maxwell_viscoelastic");
    GEO_API_END
}

int geo_update_stresses_maxwell(geo_ctx* ctx, const geo_mesh* mesh, double E, double nu, double mu,
                                const double* u_n, const double* u_next, double dt, const double* stress_n,
                                double* stress_next) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && u_n && u_next && stress_n && stress_next, "NULL argument");
    check_material(E, nu, mu);
    GEO_CHECK_ARG(dt >= 0.0, "time step must be >= 0");
    cudaStream_t s = ctx->stream;
    const int64_t n = 3 * mesh->n_nodes, ne = mesh->n_elem;
    double* out = ctx_scratch<double>(ctx, SCR_OUT0, (size_t)(6 * ne));
    const double* dun = stage_in(ctx, SCR_IN0, u_n, (size_t)n);
    const double* dunx = stage_in(ctx, SCR_IN1, u_next, (size_t)n);
    const double* dsn = stage_in(ctx, SCR_IN2, stress_n, (size_t)(6 * ne));
    const double G = E / (2.0 * (1.0 + nu));
    const double tau = mu / G;
    const double lam = E / (3.0 * (1.0 - 2.0 * nu)) - 2.0 * G / 3.0;
    reset_dev_err(ctx);
    k_maxwell_update<<<nb(ne), 128, 0, s>>>(mesh->xyz.p, mesh->conn.p, mesh->n_nodes, ne, G, lam,
                                            1.0 / (1.0 + dt / tau), dun, dunx, dsn, out, ctx->dev_err.p);
    check_launch(ctx, "k_maxwell_update");
    raise_dev_err(ctx, read_dev_err(ctx), "maxwell stress update");
    copy_out(stress_next, out, (size_t)(6 * ne), s);
    sync(ctx, "geo_update_stresses_maxwell");
    GEO_API_END
}

}  // extern "C"
