// Neumann (flux) boundary conditions on Tet10 faces, the drop-in for
// Tet10Face::from_element_face / area / integrate_flux (fem/boundary.rs:89-266),
// Assembler::find_boundary_faces (fem/assembly.rs:287-309) and
// Assembler::apply_neumann_bcs (fem/assembly.rs:248-274).
//
// One thread per face integrates the 6-node triangle with the reference's
// 3-point rule in FP64. The accumulation into f is deterministic: the 6
// contributions of every face are sorted by node with a stable radix sort and
// summed per node in face order by one thread per node, then added to f.
// Boundary faces are found on the GPU from a per-node condition mask and
// compacted in (element, local face) order, the reference's loop order.
#include <cub/cub.cuh>

#include "objects.h"

namespace geo {
namespace {

// Local face f of a Tet10 (opposite vertex f): its 3 vertices then its 3 edge
// midpoints, in the order of boundary.rs:91-127 (the face node order defines
// which triangle shape function multiplies which node).
__constant__ int kFaceNodes[4][6] = {
    {1, 2, 3, 5, 9, 8},
    {0, 2, 3, 6, 9, 7},
    {0, 1, 3, 4, 8, 7},
    {0, 1, 2, 4, 5, 6},
};

// 3-point rule on the reference triangle: (L1, L2, weight), weights summing to 1/2
__constant__ double kTri[3][3] = {
    {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0},
    {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
    {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0},
};

inline unsigned nb(int64_t n, int bs = 256) { return (unsigned)std::max<int64_t>(1, cdiv(n, bs)); }

// Quadratic triangle in area coordinates (L1, L2, L3 = 1 - L1 - L2): N and dN/dL1, dN/dL2
__device__ __forceinline__ void tri6(double l1, double l2, double (&N)[6], double (&d1)[6], double (&d2)[6]) {
    const double l3 = 1.0 - l1 - l2;
    N[0] = l1 * (2.0 * l1 - 1.0);
    N[1] = l2 * (2.0 * l2 - 1.0);
    N[2] = l3 * (2.0 * l3 - 1.0);
    N[3] = 4.0 * l1 * l2;
    N[4] = 4.0 * l2 * l3;
    N[5] = 4.0 * l3 * l1;
    d1[0] = 4.0 * l1 - 1.0;
    d2[0] = 0.0;
    d1[1] = 0.0;
    d2[1] = 4.0 * l2 - 1.0;
    d1[2] = -4.0 * l3 + 1.0;
    d2[2] = -4.0 * l3 + 1.0;
    d1[3] = 4.0 * l2;
    d2[3] = 4.0 * l1;
    d1[4] = -4.0 * l2;
    d2[4] = 4.0 * (l3 - l2);
    d1[5] = 4.0 * (l3 - l1);
    d2[5] = -4.0 * l1;
}

// Loads the 6 face nodes (ids and coordinates) of face k; false on a bad face id.
__device__ __forceinline__ bool load_face(const double* __restrict__ xyz, const int32_t* __restrict__ conn,
                                          int64_t N, int64_t E, const int32_t* __restrict__ faces, int64_t k,
                                          int32_t (&nd)[6], double (&c)[6][3]) {
    const int32_t e = faces[2 * k], lf = faces[2 * k + 1];
    if (e < 0 || e >= E || lf < 0 || lf > 3) return false;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        nd[i] = conn[(int64_t)kFaceNodes[lf][i] * E + e];
        c[i][0] = xyz[nd[i]];
        c[i][1] = xyz[N + nd[i]];
        c[i][2] = xyz[2 * N + nd[i]];
    }
    return true;
}

// |dx/dL1 x dx/dL2|
__device__ __forceinline__ double surface_jacobian(const double (&c)[6][3], const double (&d1)[6],
                                                   const double (&d2)[6]) {
    double a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            a[k] += c[i][k] * d1[i];
            b[k] += c[i][k] * d2[i];
        }
    const double x = a[1] * b[2] - a[2] * b[1], y = a[2] * b[0] - a[0] * b[2], z = a[0] * b[1] - a[1] * b[0];
    return sqrt(x * x + y * y + z * z);
}

// fe[k][i] = sum_q w_q N_i flux_k |J_q| (integrate_flux); optionally the face's node ids
__global__ void k_face_flux(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N, int64_t E,
                            int64_t nf, const int32_t* __restrict__ faces, const double* __restrict__ flux_f,
                            double flux, double* __restrict__ fe, int32_t* __restrict__ nodes_out, int* err) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nf) return;
    int32_t nd[6];
    double c[6][3];
    if (!load_face(xyz, conn, N, E, faces, k, nd, c)) {
        atomicOr(err, DEV_ERR_BOUNDS);
        return;
    }
    const double q = flux_f ? flux_f[k] : flux;
    double f[6] = {0, 0, 0, 0, 0, 0};
    for (int p = 0; p < 3; ++p) {
        double Nq[6], d1[6], d2[6];
        tri6(kTri[p][0], kTri[p][1], Nq, d1, d2);
        const double dj = surface_jacobian(c, d1, d2);
#pragma unroll
        for (int i = 0; i < 6; ++i) f[i] += kTri[p][2] * Nq[i] * q * dj;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        fe[6 * k + i] = f[i];
        if (nodes_out) nodes_out[6 * k + i] = nd[i];
    }
}

// area (Tet10Face::area)
__global__ void k_face_area(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N, int64_t E,
                            int64_t nf, const int32_t* __restrict__ faces, double* __restrict__ area, int* err) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nf) return;
    int32_t nd[6];
    double c[6][3];
    if (!load_face(xyz, conn, N, E, faces, k, nd, c)) {
        atomicOr(err, DEV_ERR_BOUNDS);
        return;
    }
    double a = 0.0;
    for (int p = 0; p < 3; ++p) {
        double Nq[6], d1[6], d2[6];
        tri6(kTri[p][0], kTri[p][1], Nq, d1, d2);
        a += kTri[p][2] * surface_jacobian(c, d1, d2);
    }
    area[k] = a;
}

// flag[4 e + f] = all 6 nodes of face f of element e satisfy the condition
__global__ void k_face_flags(const int32_t* __restrict__ conn, int64_t E, const uint8_t* __restrict__ mask,
                             uint8_t* __restrict__ flag) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 4 * E) return;
    const int64_t e = t >> 2;
    const int f = (int)(t & 3);
    bool all = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) all = all && mask[conn[(int64_t)kFaceNodes[f][i] * E + e]] != 0;
    flag[t] = all ? 1 : 0;
}

// faces[2 j] = element, faces[2 j + 1] = local face of the j-th flagged face
__global__ void k_face_pairs(const int32_t* __restrict__ sel, int64_t n, int32_t* __restrict__ faces) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    faces[2 * j] = sel[j] >> 2;
    faces[2 * j + 1] = sel[j] & 3;
}

__global__ void k_iota32(int32_t* v, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

// One thread per run of equal keys in the sorted contribution list: sums the run
// in order and adds it to f[node].
__global__ void k_run_sums(const int32_t* __restrict__ key, const int32_t* __restrict__ idx,
                           const double* __restrict__ contrib, int64_t m, int64_t n_f, double* __restrict__ f,
                           int* err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m || (i > 0 && key[i] == key[i - 1])) return;
    const int32_t node = key[i];
    double s = 0.0;
    for (int64_t j = i; j < m && key[j] == node; ++j) s += contrib[idx[j]];
    if (node < 0 || node >= n_f) {
        atomicOr(err, DEV_ERR_BOUNDS);
        return;
    }
    f[node] += s;
}

const int32_t* stage_faces(const int32_t* faces, int64_t nf, DevBuf<int32_t>& tmp, cudaStream_t s) {
    return stage_in(faces, (size_t)(2 * nf), tmp, s);
}

void check_faces(geo_ctx* ctx, const char* what) {
    check_launch(ctx, what);
    const int e = read_dev_err(ctx);
    if (e & DEV_ERR_BOUNDS) fail(GEO_ERR_INVALID_ARG, std::string(what) + ": face with an element id out of range "
                                                                         "or a local face outside 0..3");
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

int geo_face_flux(geo_ctx* ctx, const geo_mesh* mesh, int64_t n_faces, const int32_t* faces, const double* flux_f,
                  double flux, double* fe) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && (faces || n_faces == 0) && (fe || n_faces == 0), "NULL argument");
    GEO_CHECK_ARG(n_faces >= 0, "n_faces must be >= 0");
    if (n_faces == 0) return GEO_OK;
    cudaStream_t s = ctx->stream;
    DevBuf<int32_t> tf;
    DevBuf<double> tq, out(6 * n_faces);
    const int32_t* df = stage_faces(faces, n_faces, tf, s);
    const double* dq = flux_f ? stage_in(flux_f, (size_t)n_faces, tq, s) : nullptr;
    reset_dev_err(ctx);
    k_face_flux<<<nb(n_faces), 256, 0, s>>>(mesh->xyz.p, mesh->conn.p, mesh->n_nodes, mesh->n_elem, n_faces, df, dq,
                                            flux, out.p, nullptr, ctx->dev_err.p);
    check_faces(ctx, "geo_face_flux");
    copy_out(fe, out.p, (size_t)(6 * n_faces), s);
    sync(ctx, "geo_face_flux");
    GEO_API_END
}

int geo_face_area(geo_ctx* ctx, const geo_mesh* mesh, int64_t n_faces, const int32_t* faces, double* area) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && (faces || n_faces == 0) && (area || n_faces == 0), "NULL argument");
    GEO_CHECK_ARG(n_faces >= 0, "n_faces must be >= 0");
    if (n_faces == 0) return GEO_OK;
    cudaStream_t s = ctx->stream;
    DevBuf<int32_t> tf;
    DevBuf<double> out(n_faces);
    const int32_t* df = stage_faces(faces, n_faces, tf, s);
    reset_dev_err(ctx);
    k_face_area<<<nb(n_faces), 256, 0, s>>>(mesh->xyz.p, mesh->conn.p, mesh->n_nodes, mesh->n_elem, n_faces, df,
                                            out.p, ctx->dev_err.p);
    check_faces(ctx, "geo_face_area");
    copy_out(area, out.p, (size_t)n_faces, s);
    sync(ctx, "geo_face_area");
    GEO_API_END
}

int geo_find_boundary_faces(geo_ctx* ctx, const geo_mesh* mesh, const uint8_t* node_mask, int64_t max_faces,
                            int32_t* faces, int64_t* n_faces) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && node_mask && n_faces, "NULL argument");
    cudaStream_t s = ctx->stream;
    const int64_t E = mesh->n_elem, NF = 4 * E;
    GEO_CHECK_ARG(NF < INT32_MAX, "too many element faces");
    DevBuf<uint8_t> tm, flag(NF);
    DevBuf<int32_t> ids(NF), sel(NF);
    DevBuf<int64_t> cnt(1);
    const uint8_t* dm = stage_in(node_mask, (size_t)mesh->n_nodes, tm, s);
    k_face_flags<<<nb(NF), 256, 0, s>>>(mesh->conn.p, E, dm, flag.p);
    k_iota32<<<nb(NF), 256, 0, s>>>(ids.p, NF);
    check_launch(ctx, "k_face_flags");
    size_t bytes = 0;
    GEO_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, ids.p, flag.p, sel.p, cnt.p, NF, s));
    DevBuf<unsigned char> tmp(bytes + 16);
    GEO_CUDA(cub::DeviceSelect::Flagged(tmp.p, bytes, ids.p, flag.p, sel.p, cnt.p, NF, s));
    int64_t n = 0;
    GEO_CUDA(cudaMemcpyAsync(&n, cnt.p, sizeof(n), cudaMemcpyDeviceToHost, s));
    sync(ctx, "geo_find_boundary_faces");
    *n_faces = n;
    if (faces && n > 0) {
        GEO_CHECK_ARG(n <= max_faces, "faces buffer too small (see n_faces)");
        DevBuf<int32_t> pairs(2 * n);
        k_face_pairs<<<nb(n), 256, 0, s>>>(sel.p, n, pairs.p);
        check_launch(ctx, "k_face_pairs");
        copy_out(faces, pairs.p, (size_t)(2 * n), s);
        sync(ctx, "geo_find_boundary_faces");
    }
    GEO_API_END
}

int geo_apply_neumann_bcs(geo_ctx* ctx, const geo_mesh* mesh, int64_t n_faces, const int32_t* faces,
                          const double* flux_f, double flux, int64_t n_f, double* f) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && f && (faces || n_faces == 0), "NULL argument");
    GEO_CHECK_ARG(n_faces >= 0 && n_f >= mesh->n_nodes, "f must hold at least one entry per node");
    if (n_faces == 0) return GEO_OK;
    GEO_CHECK_ARG(6 * n_faces < INT32_MAX, "too many faces");
    cudaStream_t s = ctx->stream;
    const int64_t m = 6 * n_faces;
    // per-call temporaries in the context scratch (this runs every step of a transient)
    const int64_t m_al = (m + 63) & ~int64_t(63);
    int32_t* keys = ctx_scratch<int32_t>(ctx, SCR_TMP0, (size_t)(4 * m_al));
    int32_t *keys2 = keys + m_al, *idx = keys2 + m_al, *idx2 = idx + m_al;
    double* contrib = ctx_scratch<double>(ctx, SCR_TMP1, (size_t)m);
    const int32_t* df = stage_in(ctx, SCR_IN0, faces, (size_t)(2 * n_faces));
    const double* dq = flux_f ? stage_in(ctx, SCR_IN1, flux_f, (size_t)n_faces) : nullptr;
    reset_dev_err(ctx);
    k_face_flux<<<nb(n_faces), 256, 0, s>>>(mesh->xyz.p, mesh->conn.p, mesh->n_nodes, mesh->n_elem, n_faces, df, dq,
                                            flux, contrib, keys, ctx->dev_err.p);
    check_faces(ctx, "geo_apply_neumann_bcs");
    k_iota32<<<nb(m), 256, 0, s>>>(idx, m);
    int bits = 1;
    while (bits < 31 && (int64_t(1) << bits) <= mesh->n_nodes) ++bits;
    size_t bytes = 0;
    GEO_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, keys2, idx, idx2, m, 0, bits, s));
    unsigned char* tmp = ctx_scratch<unsigned char>(ctx, SCR_TMP2, bytes + 16);
    GEO_CUDA(cub::DeviceRadixSort::SortPairs(tmp, bytes, keys, keys2, idx, idx2, m, 0, bits, s));
    double* dst = f;
    if (!is_device_ptr(f)) {
        dst = ctx_scratch<double>(ctx, SCR_OUT0, (size_t)n_f);
        GEO_CUDA(cudaMemcpyAsync(dst, f, n_f * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    k_run_sums<<<nb(m), 256, 0, s>>>(keys2, idx2, contrib, m, n_f, dst, ctx->dev_err.p);
    check_faces(ctx, "geo_apply_neumann_bcs");
    if (dst != f) copy_out(f, dst, (size_t)n_f, s);
    sync(ctx, "geo_apply_neumann_bcs");
    GEO_API_END
}

}  // extern "C"
