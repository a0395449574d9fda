// Context, mesh and DOF-manager objects of the C ABI.
#include <cstdio>

#include "objects.h"

namespace geo {

void check_launch(geo_ctx* ctx, const char* what) {
    (void)ctx;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(GEO_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void sync(geo_ctx* ctx, const char* what) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) fail(GEO_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void reset_dev_err(geo_ctx* ctx) {
    GEO_CUDA(cudaMemsetAsync(ctx->dev_err.p, 0, sizeof(int), ctx->stream));
}

int read_dev_err(geo_ctx* ctx) {
    int h = 0;
    GEO_CUDA(cudaMemcpyAsync(&h, ctx->dev_err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx, "read device error word");
    return h;
}

void raise_dev_err(geo_ctx* ctx, int bits, const char* what) {
    if (bits & DEV_ERR_SINGULAR)
        fail(GEO_ERR_SINGULAR_JACOBIAN, std::string(what) + ": Singular Jacobian");
    if (bits & DEV_ERR_TIMEOUT)
        fail(GEO_ERR_TIMEOUT, std::string(what) + ": device-side wait timed out");
    if (bits & DEV_ERR_BOUNDS) fail(GEO_ERR_INVALID_ARG, std::string(what) + ": index out of range");
    (void)ctx;
}

namespace {

__global__ void aos_to_soa3(const double* __restrict__ aos, double* __restrict__ soa, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        soa[i] = aos[3 * i];
        soa[n + i] = aos[3 * i + 1];
        soa[2 * n + i] = aos[3 * i + 2];
    }
}

// mask[i] = mask[i] != 0, and the count of ones added to *count
__global__ void k_normalize_mask(uint8_t* __restrict__ mask, int64_t n, unsigned long long* __restrict__ count) {
    unsigned c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t v = mask[i] ? 1 : 0;
        mask[i] = v;
        c += v;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

__global__ void conn_to_soa(const int32_t* __restrict__ aos, int32_t* __restrict__ soa, int64_t E,
                            int64_t n_nodes, int* err) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int l = 0; l < 10; ++l) {
            const int32_t v = aos[10 * e + l];
            if (v < 0 || v >= n_nodes) atomicOr(err, DEV_ERR_BOUNDS);
            soa[l * E + e] = v;
        }
    }
}

}  // namespace

void ctx_retain(geo_ctx* c) { c->refs.fetch_add(1, std::memory_order_relaxed); }

void ctx_release(geo_ctx* c) {
    if (c->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
    int cur = -1;
    cudaGetDevice(&cur);
    const int dev = c->device;
    cudaSetDevice(dev);
    cudaStreamSynchronize(c->stream);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    dev_release_cached(dev);
    if (cur >= 0 && cur != dev) cudaSetDevice(cur);
}
}  // namespace geo

using namespace geo;

extern "C" {

const char* geo_version(void) { return "geofem-b200 0.1 (sm_100a)"; }

int geo_device_count(int* count) {
    GEO_API_BEGIN(nullptr)
    GEO_CHECK_ARG(count, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    GEO_API_END
}

int geo_ctx_create(int device, geo_ctx** out) {
    GEO_API_BEGIN(nullptr)
    GEO_CHECK_ARG(out, "out is NULL");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        fail(GEO_ERR_NO_DEVICE, "no CUDA device visible");
    }
    GEO_CHECK_ARG(device >= 0 && device < n, "device ordinal out of range");
    GEO_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    GEO_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        fail(GEO_ERR_UNSUPPORTED, "libgeofem is built for sm_100a (B200); device is sm_" +
                                      std::to_string(prop.major) + std::to_string(prop.minor));
    auto ctx = std::make_unique<geo_ctx>();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    GEO_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    GEO_CUDA(cudaEventCreate(&ctx->ev0));
    GEO_CUDA(cudaEventCreate(&ctx->ev1));
    ctx->dev_err.alloc(4);
    GEO_CUDA(cudaMemset(ctx->dev_err.p, 0, 4 * sizeof(int)));
    *out = ctx.release();
    GEO_API_END
}

int geo_ctx_destroy(geo_ctx* ctx) {
    if (!ctx) return GEO_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    geo::ctx_release(ctx);  // freed now, or when the last object made on it is destroyed
    return GEO_OK;
}

const char* geo_last_error(const geo_ctx* ctx) {
    return ctx ? ctx->err.c_str() : geo::g_thread_err.c_str();
}

int geo_sm_count(const geo_ctx* ctx, int* sm_count) {
    if (!ctx || !sm_count) return GEO_ERR_INVALID_ARG;
    *sm_count = ctx->sm_count;
    return GEO_OK;
}

int geo_ctx_stream(const geo_ctx* ctx, void** stream) {
    if (!ctx || !stream) return GEO_ERR_INVALID_ARG;
    *stream = (void*)ctx->stream;
    return GEO_OK;
}

int geo_mesh_create(geo_ctx* ctx, int64_t n_nodes, const double* xyz, int64_t n_elem,
                    const int32_t* conn, geo_mesh** out) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && out, "ctx/out is NULL");
    GEO_CHECK_ARG(n_nodes > 0 && n_nodes < (int64_t(1) << 31), "n_nodes out of range");
    GEO_CHECK_ARG(n_elem > 0 && n_elem * 10 < (int64_t(1) << 31), "n_elem out of range");
    GEO_CHECK_ARG(xyz && conn, "xyz/conn is NULL");
    auto m = std::make_unique<geo_mesh>();
    m->ctx = ctx;
    m->ref.set(ctx);
    m->n_nodes = n_nodes;
    m->n_elem = n_elem;
    cudaStream_t s = ctx->stream;
    DevBuf<double> txyz;
    DevBuf<int32_t> tconn;
    const double* dxyz = stage_in(xyz, 3 * n_nodes, txyz, s);
    const int32_t* dconn = stage_in(conn, 10 * n_elem, tconn, s);
    m->xyz.alloc(3 * n_nodes);
    m->conn.alloc(10 * n_elem);
    reset_dev_err(ctx);
    aos_to_soa3<<<std::min<int64_t>(cdiv(n_nodes, 256), 65535), 256, 0, s>>>(dxyz, m->xyz.p, n_nodes);
    check_launch(ctx, "aos_to_soa3");
    conn_to_soa<<<std::min<int64_t>(cdiv(n_elem, 256), 65535), 256, 0, s>>>(dconn, m->conn.p, n_elem,
                                                                             n_nodes, ctx->dev_err.p);
    check_launch(ctx, "conn_to_soa");
    const int bits = read_dev_err(ctx);
    if (bits & DEV_ERR_BOUNDS) fail(GEO_ERR_INVALID_ARG, "connectivity references a node id out of range");
    *out = m.release();
    GEO_API_END
}

int geo_mesh_destroy(geo_mesh* mesh) {
    if (!mesh) return GEO_OK;
    cudaSetDevice(mesh->ctx->device);
    delete mesh;
    return GEO_OK;
}

int geo_dofs_create(geo_ctx* ctx, int64_t n_nodes, int32_t dofs_per_node, const uint8_t* mask,
                    const double* values, geo_dofs** out) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && out, "ctx/out is NULL");
    GEO_CHECK_ARG(n_nodes > 0, "n_nodes must be positive");
    GEO_CHECK_ARG(dofs_per_node >= 1 && dofs_per_node <= 3, "dofs_per_node must be 1..3");
    auto d = std::make_unique<geo_dofs>();
    d->ctx = ctx;
    d->ref.set(ctx);
    d->n_nodes = n_nodes;
    d->dpn = dofs_per_node;
    d->n_dofs = n_nodes * dofs_per_node;
    GEO_CHECK_ARG(d->n_dofs < (int64_t(1) << 31), "too many DOFs");
    // copied straight to the device (DMA from pinned callers' buffers); the mask is
    // normalised to 0/1 and its Dirichlet DOFs counted there
    cudaStream_t s = ctx->stream;
    d->mask.alloc(d->n_dofs);
    d->vals.alloc(d->n_dofs);
    if (mask) GEO_CUDA(cudaMemcpyAsync(d->mask.p, mask, d->n_dofs, cudaMemcpyDefault, s));
    else GEO_CUDA(cudaMemsetAsync(d->mask.p, 0, d->n_dofs, s));
    if (values) GEO_CUDA(cudaMemcpyAsync(d->vals.p, values, d->n_dofs * sizeof(double), cudaMemcpyDefault, s));
    else GEO_CUDA(cudaMemsetAsync(d->vals.p, 0, d->n_dofs * sizeof(double), s));
    unsigned long long* cnt = ctx_scratch<unsigned long long>(ctx, SCR_TMP0, 1);
    GEO_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
    k_normalize_mask<<<(unsigned)std::min<int64_t>(cdiv(d->n_dofs, 256), (int64_t)ctx->sm_count * 8), 256, 0, s>>>(
        d->mask.p, d->n_dofs, cnt);
    check_launch(ctx, "k_normalize_mask");
    unsigned long long nd = 0;
    GEO_CUDA(cudaMemcpyAsync(&nd, cnt, sizeof nd, cudaMemcpyDeviceToHost, s));
    GEO_CUDA(cudaStreamSynchronize(s));
    d->n_dir = (int64_t)nd;
    *out = d.release();
    GEO_API_END
}

int geo_dofs_num_dirichlet(const geo_dofs* dofs, int64_t* count) {
    if (!dofs || !count) return GEO_ERR_INVALID_ARG;
    *count = dofs->n_dir;
    return GEO_OK;
}

int geo_dofs_destroy(geo_dofs* dofs) {
    if (!dofs) return GEO_OK;
    cudaSetDevice(dofs->ctx->device);
    delete dofs;
    return GEO_OK;
}

}  // extern "C"
