// K2/K3: deterministic CSR assembly and Dirichlet elimination (FP64).
//
// The reference collects 100 (900) triplets per element and lets sprs sort and
// merge them (assembly.rs:69-117, :389-437). Here a node -> (element, local)
// inverse map, sorted by element, drives everything:
//   * the sparsity pattern of row i is the sorted union of the nodes of the
//     elements incident to node i (one warp per row, bitonic sort in shared
//     memory) -- identical to sprs' sorted, merged structure;
//   * each row sums its contributions in ascending element order, the order in
//     which the reference's triplets reach every (row, col) entry;
//   * load vectors gather per node in the same order (assembly.rs:130-154).
// No atomics touch values, so every result is bit-reproducible run to run.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>

#include "objects.h"
#include "tet10.cuh"

namespace geo {

void element_thermal_stiffness(geo_ctx* ctx, const geo_mesh* m, const double* k_e_dev, double k, double* out);
void element_thermal_load(geo_ctx* ctx, const geo_mesh* m, double Q, double* out);
void element_elasticity_stiffness(geo_ctx* ctx, const geo_mesh* m, const double* E_dev, double E, double nu,
                                  double* out);
void element_gravity_load(geo_ctx* ctx, const geo_mesh* m, double rho, const double g[3], double* out);

namespace {

constexpr int kPatCap = 1024;  // candidate columns per node row (10 x incident elements)
constexpr int kPatWarps = 4;

inline unsigned blocks(int64_t n, int bs) { return (unsigned)std::max<int64_t>(1, cdiv(n, bs)); }

template <class T>
void exclusive_scan(const T* in, T* out, int64_t n, cudaStream_t s) {
    size_t tmp_bytes = 0;
    GEO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, n, s));
    DevBuf<unsigned char> tmp(tmp_bytes + 16);
    GEO_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, in, out, n, s));
    GEO_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------- inverse map
__global__ void k_inc_count(const int32_t* __restrict__ conn, int64_t E, int32_t* __restrict__ cnt) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= E * 10) return;
    atomicAdd(&cnt[conn[t]], 1);  // conn is SoA [10][E]; t = l*E + e
}

__global__ void k_inc_fill(const int32_t* __restrict__ conn, int64_t E, const int32_t* __restrict__ ptr,
                           int32_t* __restrict__ cursor, int32_t* __restrict__ inc) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= E * 10) return;
    const int64_t l = t / E, e = t % E;
    const int32_t n = conn[t];
    const int32_t pos = ptr[n] + atomicAdd(&cursor[n], 1);
    inc[pos] = (int32_t)(e * 10 + l);
}

// Sorts every node's incidence segment ascending (element-major) by insertion sort.
__global__ void k_inc_sort(const int32_t* __restrict__ ptr, int32_t* __restrict__ inc, int64_t N) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int32_t b = ptr[i], e = ptr[i + 1];
    for (int32_t p = b + 1; p < e; ++p) {
        const int32_t v = inc[p];
        int32_t q = p - 1;
        while (q >= b && inc[q] > v) {
            inc[q + 1] = inc[q];
            --q;
        }
        inc[q + 1] = v;
    }
}

// ---------------------------------------------------------------- node pattern
// One warp per node row: gather candidate columns, bitonic sort, count / emit
// the distinct ones. err gets DEV_ERR_BOUNDS when a row exceeds kPatCap.
__global__ void __launch_bounds__(32 * kPatWarps)
k_pattern(const int32_t* __restrict__ conn, int64_t E, const int32_t* __restrict__ ptr,
          const int32_t* __restrict__ inc, int64_t N, int64_t* __restrict__ row_cnt,
          const int64_t* __restrict__ out_ptr, int32_t* __restrict__ out_idx, int* err) {
    __shared__ int32_t sbuf[kPatWarps][kPatCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t* buf = sbuf[w];
    const int64_t nwarps = (int64_t)gridDim.x * kPatWarps;
    for (int64_t i = blockIdx.x * (int64_t)kPatWarps + w; i < N; i += nwarps) {
        const int32_t b = ptr[i];
        const int deg = ptr[i + 1] - b;
        const int nc = 10 * deg;
        if (nc > kPatCap) {
            if (lane == 0) {
                atomicOr(err, DEV_ERR_BOUNDS);
                if (row_cnt) row_cnt[i] = 0;
            }
            continue;
        }
        int P = 32;
        while (P < nc) P <<= 1;
        for (int t = lane; t < P; t += 32) {
            int32_t v = INT_MAX;
            if (t < nc) {
                const int32_t el = inc[b + t / 10];
                v = conn[(int64_t)(t % 10) * E + el / 10];
            }
            buf[t] = v;
        }
        __syncwarp();
        for (int k = 2; k <= P; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int t = lane; t < P; t += 32) {
                    const int ixj = t ^ j;
                    if (ixj > t) {
                        const int32_t a = buf[t], c = buf[ixj];
                        const bool up = (t & k) == 0;
                        if ((a > c) == up) {
                            buf[t] = c;
                            buf[ixj] = a;
                        }
                    }
                }
                __syncwarp();
            }
        int64_t run = 0;
        const int64_t base = out_idx ? out_ptr[i] : 0;
        for (int t0 = 0; t0 < P; t0 += 32) {
            const int t = t0 + lane;
            const int32_t v = buf[t];
            const bool uniq = v != INT_MAX && (t == 0 || buf[t - 1] != v);
            const unsigned bal = __ballot_sync(0xffffffffu, uniq);
            if (out_idx && uniq) out_idx[base + run + __popc(bal & ((1u << lane) - 1u))] = v;
            run += __popc(bal);
        }
        if (row_cnt && lane == 0) row_cnt[i] = run;
        __syncwarp();
    }
}

__device__ __forceinline__ int64_t find_col(const int32_t* __restrict__ idx, int64_t b, int64_t e, int32_t c) {
    // lower_bound on the sorted column list [b, e)
    while (b < e) {
        const int64_t m = (b + e) >> 1;
        if (idx[m] < c) b = m + 1;
        else e = m;
    }
    return b;
}

// ---------------------------------------------------------------- values
__global__ void k_thermal_values(const int32_t* __restrict__ conn, int64_t E, const int32_t* __restrict__ ptr,
                                 const int32_t* __restrict__ inc, const int64_t* __restrict__ pptr,
                                 const int32_t* __restrict__ pidx, const double* __restrict__ Ke, int64_t N,
                                 double* __restrict__ data) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int64_t rb = pptr[i], re = pptr[i + 1];
    for (int32_t p = ptr[i]; p < ptr[i + 1]; ++p) {
        const int32_t el = inc[p];
        const int64_t e = el / 10;
        const int l = el % 10;
        const double* ke = Ke + e * 100 + l * 10;
        for (int j = 0; j < 10; ++j) {
            const int32_t c = conn[(int64_t)j * E + e];
            const int64_t pos = find_col(pidx, rb, re, c);
            data[pos] = __dadd_rn(data[pos], ke[j]);
        }
    }
}

// rows (i, a) of the 3-DOF system; node pattern row i expanded by 3x3 blocks
__global__ void k_elastic_structure(const int64_t* __restrict__ pptr, const int32_t* __restrict__ pidx,
                                    int64_t N, int64_t* __restrict__ indptr, int32_t* __restrict__ indices) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int64_t i = t / 3;
    const int a = (int)(t % 3);
    const int64_t L = pptr[i + 1] - pptr[i];
    const int64_t row0 = 9 * pptr[i] + a * 3 * L;
    indptr[t] = row0;
    if (t == 3 * N - 1) indptr[3 * N] = 9 * pptr[N];
    for (int64_t p = 0; p < L; ++p) {
        const int32_t c = pidx[pptr[i] + p];
#pragma unroll
        for (int b = 0; b < 3; ++b) indices[row0 + 3 * p + b] = 3 * c + b;
    }
}

__global__ void k_elastic_values(const int32_t* __restrict__ conn, int64_t E, const int32_t* __restrict__ ptr,
                                 const int32_t* __restrict__ inc, const int64_t* __restrict__ pptr,
                                 const int32_t* __restrict__ pidx, const double* __restrict__ Ke, int64_t N,
                                 double* __restrict__ data) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int64_t i = t / 3;
    const int a = (int)(t % 3);
    const int64_t rb = pptr[i], re = pptr[i + 1];
    const int64_t row0 = 9 * rb + a * 3 * (re - rb);
    for (int32_t p = ptr[i]; p < ptr[i + 1]; ++p) {
        const int32_t el = inc[p];
        const int64_t e = el / 10;
        const int l = el % 10;
        const double* ke = Ke + e * 900 + (3 * l + a) * 30;
        for (int j = 0; j < 10; ++j) {
            const int32_t c = conn[(int64_t)j * E + e];
            const int64_t pos = find_col(pidx, rb, re, c) - rb;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                double* d = data + row0 + 3 * pos + b;
                *d = __dadd_rn(*d, ke[3 * j + b]);
            }
        }
    }
}

// f_{dpn*i + a} = sum over incidences (element order) of fe[e][dpn*l + a]
__global__ void k_gather_load(const int32_t* __restrict__ ptr, const int32_t* __restrict__ inc,
                              const double* __restrict__ fe, int64_t N, int dpn, double* __restrict__ f) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= dpn * N) return;
    const int64_t i = t / dpn;
    const int a = (int)(t % dpn);
    double s = 0.0;
    for (int32_t p = ptr[i]; p < ptr[i + 1]; ++p) {
        const int32_t el = inc[p];
        s = __dadd_rn(s, fe[(int64_t)(el / 10) * (10 * dpn) + dpn * (el % 10) + a]);
    }
    f[t] = s;
}

// ---------------------------------------------------------------- Dirichlet
__global__ void k_max_abs_diag(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                               const double* __restrict__ data, int64_t n, unsigned long long* out) {
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = find_col(indices, indptr[i], indptr[i + 1], (int32_t)i);
        if (p < indptr[i + 1] && indices[p] == i) m = fmax(m, fabs(data[p]));
    }
    // non-negative doubles order like their bit patterns
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_dirichlet_rhs(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                const double* __restrict__ data, const uint8_t* __restrict__ mask,
                                const double* __restrict__ g, const double* __restrict__ f, double cd, int64_t n,
                                double* __restrict__ fbc, int64_t* __restrict__ rowcnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mask[i]) {
        fbc[i] = __dmul_rn(g[i], cd);
        rowcnt[i] = 1;
        return;
    }
    double s = f[i];
    int64_t c = 0;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
        const int32_t j = indices[p];
        if (mask[j]) s = __dsub_rn(s, __dmul_rn(data[p], g[j]));
        else ++c;
    }
    fbc[i] = s;
    rowcnt[i] = c;
}

__global__ void k_dirichlet_fill(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                 const double* __restrict__ data, const uint8_t* __restrict__ mask, double cd,
                                 int64_t n, const int64_t* __restrict__ optr, int32_t* __restrict__ oidx,
                                 double* __restrict__ odata) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t o = optr[i];
    if (mask[i]) {
        oidx[o] = (int32_t)i;
        odata[o] = cd;
        return;
    }
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
        const int32_t j = indices[p];
        if (!mask[j]) {
            oidx[o] = j;
            odata[o] = data[p];
            ++o;
        }
    }
}

__global__ void k_set_last(int64_t* ptr, int64_t n, const int64_t* cnt) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ptr[n] = ptr[n - 1] + cnt[n - 1];
}

// ---------------------------------------------------------------- SpMV
template <int VEC>
__global__ void k_spmv(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                       const double* __restrict__ data, const double* __restrict__ x, int64_t n,
                       double* __restrict__ y) {
    const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t row = gt / VEC;
    const int sub = (int)(gt % VEC);
    if (row >= n) return;
    double s = 0.0;
    for (int64_t p = indptr[row] + sub; p < indptr[row + 1]; p += VEC) s += data[p] * x[indices[p]];
#pragma unroll
    for (int o = VEC / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, VEC);
    if (sub == 0) y[row] = s;
}

}  // namespace

// ---------------------------------------------------------------- shared builders
void ensure_inverse_map(geo_mesh* m) {
    if (m->inc.p) return;
    geo_ctx* ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    const int64_t N = m->n_nodes, E = m->n_elem;
    DevBuf<int32_t> cnt(N + 1), cursor(N);
    GEO_CUDA(cudaMemsetAsync(cnt.p, 0, (N + 1) * sizeof(int32_t), s));
    GEO_CUDA(cudaMemsetAsync(cursor.p, 0, N * sizeof(int32_t), s));
    k_inc_count<<<blocks(E * 10, 256), 256, 0, s>>>(m->conn.p, E, cnt.p);
    check_launch(ctx, "k_inc_count");
    m->inc_ptr.alloc(N + 1);
    exclusive_scan(cnt.p, m->inc_ptr.p, N + 1, s);
    m->inc.alloc(E * 10);
    k_inc_fill<<<blocks(E * 10, 256), 256, 0, s>>>(m->conn.p, E, m->inc_ptr.p, cursor.p, m->inc.p);
    check_launch(ctx, "k_inc_fill");
    k_inc_sort<<<blocks(N, 128), 128, 0, s>>>(m->inc_ptr.p, m->inc.p, N);
    check_launch(ctx, "k_inc_sort");
    sync(ctx, "inverse map");
}

void ensure_pattern(geo_mesh* m) {
    if (m->pat_nnz >= 0) return;
    ensure_inverse_map(m);
    geo_ctx* ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    const int64_t N = m->n_nodes, E = m->n_elem;
    DevBuf<int64_t> cnt(N + 1);
    GEO_CUDA(cudaMemsetAsync(cnt.p, 0, (N + 1) * sizeof(int64_t), s));
    reset_dev_err(ctx);
    const unsigned g = (unsigned)std::min<int64_t>(cdiv(N, kPatWarps), 1 << 20);
    k_pattern<<<g, 32 * kPatWarps, 0, s>>>(m->conn.p, E, m->inc_ptr.p, m->inc.p, N, cnt.p, nullptr, nullptr,
                                           ctx->dev_err.p);
    check_launch(ctx, "k_pattern(count)");
    if (read_dev_err(ctx) & DEV_ERR_BOUNDS)
        fail(GEO_ERR_UNSUPPORTED, "a node is shared by more than 102 elements (row pattern buffer)");
    m->pat_ptr.alloc(N + 1);
    exclusive_scan(cnt.p, m->pat_ptr.p, N + 1, s);
    int64_t nnz = 0;
    GEO_CUDA(cudaMemcpy(&nnz, m->pat_ptr.p + N, sizeof(int64_t), cudaMemcpyDeviceToHost));
    m->pat_idx.alloc(nnz);
    k_pattern<<<g, 32 * kPatWarps, 0, s>>>(m->conn.p, E, m->inc_ptr.p, m->inc.p, N, nullptr, m->pat_ptr.p,
                                           m->pat_idx.p, ctx->dev_err.p);
    check_launch(ctx, "k_pattern(fill)");
    sync(ctx, "pattern");
    m->pat_nnz = nnz;
}

void csr_spmv(geo_ctx* ctx, const geo_csr* A, const double* x, double* y) {
    const int64_t n = A->n_rows;
    k_spmv<8><<<blocks(n * 8, 256), 256, 0, ctx->stream>>>(A->indptr.p, A->indices.p, A->data.p, x, n, y);
    check_launch(ctx, "k_spmv");
}

}  // namespace geo

using namespace geo;

namespace {

std::unique_ptr<geo_csr> new_csr(geo_ctx* ctx, int64_t rows, int64_t cols, int64_t nnz) {
    auto A = std::make_unique<geo_csr>();
    A->ctx = ctx;
    A->ref.set(ctx);
    A->n_rows = rows;
    A->n_cols = cols;
    A->nnz = nnz;
    A->indptr.alloc(rows + 1);
    A->indices.alloc(std::max<int64_t>(nnz, 1));
    A->data.alloc(std::max<int64_t>(nnz, 1));
    return A;
}

void deliver(geo_ctx* ctx, double* out, const double* dev, size_t n) {
    copy_out(out, dev, n, ctx->stream);
    sync(ctx, "deliver");
}

}  // namespace

extern "C" {

int geo_assemble_thermal_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, const double* k_e,
                                   double k, geo_csr** K) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && K, "NULL argument");
    GEO_CHECK_ARG(!dofs || (dofs->dpn == 1 && dofs->n_nodes == mesh->n_nodes),
                  "thermal assembly needs 1 DOF per node on the same node set");
    geo_mesh* m = const_cast<geo_mesh*>(mesh);
    ensure_pattern(m);
    cudaStream_t s = ctx->stream;
    const int64_t N = m->n_nodes, E = m->n_elem;
    DevBuf<double> tk, Ke(E * 100);
    const double* dk = k_e ? stage_in(k_e, E, tk, s) : nullptr;
    reset_dev_err(ctx);
    element_thermal_stiffness(ctx, m, dk, k, Ke.p);
    raise_dev_err(ctx, read_dev_err(ctx), "thermal stiffness");
    auto A = new_csr(ctx, N, N, m->pat_nnz);
    GEO_CUDA(cudaMemcpyAsync(A->indptr.p, m->pat_ptr.p, (N + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
    GEO_CUDA(cudaMemcpyAsync(A->indices.p, m->pat_idx.p, m->pat_nnz * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    GEO_CUDA(cudaMemsetAsync(A->data.p, 0, m->pat_nnz * sizeof(double), s));
    k_thermal_values<<<blocks(N, 128), 128, 0, s>>>(m->conn.p, E, m->inc_ptr.p, m->inc.p, m->pat_ptr.p,
                                                     m->pat_idx.p, Ke.p, N, A->data.p);
    check_launch(ctx, "k_thermal_values");
    sync(ctx, "assemble thermal stiffness");
    *K = A.release();
    GEO_API_END
}

int geo_assemble_thermal_load(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, double source,
                              double* f) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && f, "NULL argument");
    GEO_CHECK_ARG(!dofs || (dofs->dpn == 1 && dofs->n_nodes == mesh->n_nodes),
                  "thermal load needs 1 DOF per node on the same node set");
    geo_mesh* m = const_cast<geo_mesh*>(mesh);
    ensure_inverse_map(m);
    cudaStream_t s = ctx->stream;
    DevBuf<double> fe(m->n_elem * 10), out(m->n_nodes);
    reset_dev_err(ctx);
    element_thermal_load(ctx, m, source, fe.p);
    k_gather_load<<<blocks(m->n_nodes, 256), 256, 0, s>>>(m->inc_ptr.p, m->inc.p, fe.p, m->n_nodes, 1, out.p);
    check_launch(ctx, "k_gather_load");
    deliver(ctx, f, out.p, m->n_nodes);
    GEO_API_END
}

int geo_assemble_elasticity_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, const double* E_e,
                                      double E, double nu, geo_csr** K) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && K, "NULL argument");
    GEO_CHECK_ARG(!dofs || dofs->dpn == 3, "Elasticity requires 3 DOF per node");
    GEO_CHECK_ARG(!dofs || dofs->n_nodes == mesh->n_nodes, "DOF manager and mesh disagree on the node count");
    GEO_CHECK_ARG(nu > -1.0 && nu < 0.5, "Poisson's ratio must be in (-1, 0.5)");
    geo_mesh* m = const_cast<geo_mesh*>(mesh);
    ensure_pattern(m);
    cudaStream_t s = ctx->stream;
    const int64_t N = m->n_nodes, Ne = m->n_elem;
    DevBuf<double> tE, Ke(Ne * 900);
    const double* dE = E_e ? stage_in(E_e, Ne, tE, s) : nullptr;
    reset_dev_err(ctx);
    element_elasticity_stiffness(ctx, m, dE, E, nu, Ke.p);
    raise_dev_err(ctx, read_dev_err(ctx), "elasticity stiffness");
    auto A = new_csr(ctx, 3 * N, 3 * N, 9 * m->pat_nnz);
    k_elastic_structure<<<blocks(3 * N, 128), 128, 0, s>>>(m->pat_ptr.p, m->pat_idx.p, N, A->indptr.p,
                                                           A->indices.p);
    check_launch(ctx, "k_elastic_structure");
    GEO_CUDA(cudaMemsetAsync(A->data.p, 0, A->nnz * sizeof(double), s));
    k_elastic_values<<<blocks(3 * N, 128), 128, 0, s>>>(m->conn.p, Ne, m->inc_ptr.p, m->inc.p, m->pat_ptr.p,
                                                        m->pat_idx.p, Ke.p, N, A->data.p);
    check_launch(ctx, "k_elastic_values");
    sync(ctx, "assemble elasticity stiffness");
    *K = A.release();
    GEO_API_END
}

int geo_assemble_gravity_load(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, double density,
                              const double gravity[3], double* f) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && f && gravity, "NULL argument");
    GEO_CHECK_ARG(!dofs || dofs->dpn == 3, "Gravity load requires 3 DOF per node");
    geo_mesh* m = const_cast<geo_mesh*>(mesh);
    ensure_inverse_map(m);
    cudaStream_t s = ctx->stream;
    DevBuf<double> fe(m->n_elem * 30), out(3 * m->n_nodes);
    element_gravity_load(ctx, m, density, gravity, fe.p);
    k_gather_load<<<blocks(3 * m->n_nodes, 256), 256, 0, s>>>(m->inc_ptr.p, m->inc.p, fe.p, m->n_nodes, 3, out.p);
    check_launch(ctx, "k_gather_load");
    deliver(ctx, f, out.p, 3 * m->n_nodes);
    GEO_API_END
}

int geo_apply_dirichlet_bcs(geo_ctx* ctx, const geo_csr* K, const double* f, const geo_dofs* dofs,
                            geo_csr** K_bc, double* f_bc) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && K && f && dofs && K_bc && f_bc, "NULL argument");
    GEO_CHECK_ARG(K->n_rows == dofs->n_dofs && K->n_cols == dofs->n_dofs, "matrix and DOF manager disagree");
    cudaStream_t s = ctx->stream;
    const int64_t n = K->n_rows;
    DevBuf<double> tf, fbc(n);
    const double* df = stage_in(f, n, tf, s);
    DevBuf<unsigned long long> mx(1);
    GEO_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(unsigned long long), s));
    k_max_abs_diag<<<blocks(std::min<int64_t>(n, 148 * 2048), 256), 256, 0, s>>>(K->indptr.p, K->indices.p,
                                                                                  K->data.p, n, mx.p);
    check_launch(ctx, "k_max_abs_diag");
    unsigned long long bits = 0;
    GEO_CUDA(cudaMemcpyAsync(&bits, mx.p, sizeof(bits), cudaMemcpyDeviceToHost, s));
    sync(ctx, "char_diag");
    double maxd;
    std::memcpy(&maxd, &bits, sizeof(double));
    const double cd = maxd > 1.0 ? maxd : 1.0;  // assembly.rs:184-193
    DevBuf<int64_t> cnt(n + 1);
    k_dirichlet_rhs<<<blocks(n, 256), 256, 0, s>>>(K->indptr.p, K->indices.p, K->data.p, dofs->mask.p,
                                                   dofs->vals.p, df, cd, n, fbc.p, cnt.p);
    check_launch(ctx, "k_dirichlet_rhs");
    DevBuf<int64_t> optr(n + 1);
    exclusive_scan(cnt.p, optr.p, n, s);
    k_set_last<<<1, 32, 0, s>>>(optr.p, n, cnt.p);
    int64_t nnz = 0;
    GEO_CUDA(cudaMemcpyAsync(&nnz, optr.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    sync(ctx, "dirichlet counts");
    auto B = new_csr(ctx, n, K->n_cols, nnz);
    GEO_CUDA(cudaMemcpyAsync(B->indptr.p, optr.p, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
    k_dirichlet_fill<<<blocks(n, 256), 256, 0, s>>>(K->indptr.p, K->indices.p, K->data.p, dofs->mask.p, cd, n,
                                                    optr.p, B->indices.p, B->data.p);
    check_launch(ctx, "k_dirichlet_fill");
    deliver(ctx, f_bc, fbc.p, n);
    *K_bc = B.release();
    GEO_API_END
}

int geo_csr_create(geo_ctx* ctx, int64_t n_rows, int64_t n_cols, int64_t nnz, const int64_t* indptr,
                   const int32_t* indices, const double* data, geo_csr** out) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && out && indptr && (nnz == 0 || (indices && data)), "NULL argument");
    GEO_CHECK_ARG(n_rows > 0 && n_cols > 0 && nnz >= 0, "bad dimensions");
    GEO_CHECK_ARG(n_rows < (int64_t(1) << 31) && n_cols < (int64_t(1) << 31), "dimensions exceed int32 indices");
    // validate structure on the host
    std::vector<int64_t> hp(n_rows + 1);
    std::vector<int32_t> hi(nnz);
    GEO_CUDA(cudaMemcpy(hp.data(), indptr, (n_rows + 1) * sizeof(int64_t), cudaMemcpyDefault));
    if (nnz) GEO_CUDA(cudaMemcpy(hi.data(), indices, nnz * sizeof(int32_t), cudaMemcpyDefault));
    GEO_CHECK_ARG(hp[0] == 0 && hp[n_rows] == nnz, "indptr must start at 0 and end at nnz");
    for (int64_t i = 0; i < n_rows; ++i) {
        GEO_CHECK_ARG(hp[i] <= hp[i + 1], "indptr must be non-decreasing");
        for (int64_t p = hp[i]; p < hp[i + 1]; ++p) {
            GEO_CHECK_ARG(hi[p] >= 0 && hi[p] < n_cols, "column index out of range");
            GEO_CHECK_ARG(p == hp[i] || hi[p - 1] < hi[p], "columns must be sorted and unique within a row");
        }
    }
    auto A = new_csr(ctx, n_rows, n_cols, nnz);
    GEO_CUDA(cudaMemcpy(A->indptr.p, hp.data(), (n_rows + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
    if (nnz) {
        GEO_CUDA(cudaMemcpy(A->indices.p, hi.data(), nnz * sizeof(int32_t), cudaMemcpyHostToDevice));
        GEO_CUDA(cudaMemcpy(A->data.p, data, nnz * sizeof(double), cudaMemcpyDefault));
    }
    *out = A.release();
    GEO_API_END
}

int geo_csr_info(const geo_csr* A, int64_t* n_rows, int64_t* n_cols, int64_t* nnz) {
    if (!A) return GEO_ERR_INVALID_ARG;
    if (n_rows) *n_rows = A->n_rows;
    if (n_cols) *n_cols = A->n_cols;
    if (nnz) *nnz = A->nnz;
    return GEO_OK;
}

int geo_csr_copy(const geo_csr* A, int64_t* indptr, int32_t* indices, double* data) {
    GEO_API_BEGIN(A ? A->ctx : nullptr)
    GEO_CHECK_ARG(A, "NULL matrix");
    cudaStream_t s = A->ctx->stream;
    if (indptr) copy_out(indptr, A->indptr.p, A->n_rows + 1, s);
    if (indices) copy_out(indices, A->indices.p, A->nnz, s);
    if (data) copy_out(data, A->data.p, A->nnz, s);
    sync(A->ctx, "csr copy");
    GEO_API_END
}

int geo_csr_device_ptrs(const geo_csr* A, const int64_t** indptr, const int32_t** indices, const double** data) {
    if (!A) return GEO_ERR_INVALID_ARG;
    if (indptr) *indptr = A->indptr.p;
    if (indices) *indices = A->indices.p;
    if (data) *data = A->data.p;
    return GEO_OK;
}

int geo_csr_apply(geo_ctx* ctx, const geo_csr* A, const double* x, double* y) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && A && x && y, "NULL argument");
    cudaStream_t s = ctx->stream;
    DevBuf<double> tx, ty(A->n_rows);
    const double* dx = stage_in(x, A->n_cols, tx, s);
    csr_spmv(ctx, A, dx, ty.p);
    deliver(ctx, y, ty.p, A->n_rows);
    GEO_API_END
}

int geo_csr_destroy(geo_csr* A) {
    if (!A) return GEO_OK;
    cudaSetDevice(A->ctx->device);
    delete A;
    return GEO_OK;
}

}  // extern "C"
