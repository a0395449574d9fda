// Internal definitions of the opaque C-ABI objects and the cross-file helpers.
#pragma once

#include <atomic>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace geo {
// Slots of a context's scratch: one per temporary that a single call keeps live.
enum ScratchSlot : int { SCR_IN0, SCR_IN1, SCR_IN2, SCR_OUT0, SCR_OUT1, SCR_TMP0, SCR_TMP1, SCR_TMP2, kScratchSlots };
}  // namespace geo

struct geo_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    std::string err;
    geo::DevBuf<int> dev_err;  // [0]: DEV_ERR_* bits of element kernels
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Grow-only scratch for the temporaries of the entry points that run every
    // step (staged inputs, per-element arrays, VTU offsets and chunks), and two
    // pinned host buffers. Calls on one context run in order on its stream, so a
    // slot is reused from call to call with no cudaMalloc or cudaFree: cudaFree
    // synchronises the device, and in processes holding several GB it stalled
    // single calls for up to a second. Held until the context is destroyed.
    geo::DevBuf<unsigned char> scratch[geo::kScratchSlots];
    geo::HostBuf<char> pinned[2];
    // references: the creator's (dropped by geo_ctx_destroy) plus one per live object
    // made on this context (meshes, DOF sets, matrices, operators)
    std::atomic<int> refs{1};
};

namespace geo {
void ctx_retain(geo_ctx* c);
// Drops one reference; the last one destroys the stream and events and frees the context.
void ctx_release(geo_ctx* c);
// The reference an object holds on the context it was made on: the context stays
// valid until the caller destroyed it and every object made on it is gone, in
// whatever order the caller (or a garbage collector) destroys them.
struct CtxRef {
    geo_ctx* c = nullptr;
    CtxRef() = default;
    CtxRef(const CtxRef&) = delete;
    CtxRef& operator=(const CtxRef&) = delete;
    void set(geo_ctx* x) {
        if (x) ctx_retain(x);
        if (c) ctx_release(c);
        c = x;
    }
    ~CtxRef() {
        if (c) ctx_release(c);
    }
};
}  // namespace geo

struct geo_mesh {
    geo_ctx* ctx = nullptr;
    geo::CtxRef ref;  // declared first after ctx: released after every buffer below
    int64_t n_nodes = 0, n_elem = 0;
    geo::DevBuf<double> xyz;       // SoA [3][N]
    geo::DevBuf<int32_t> conn;     // SoA [10][E]
    // node -> (element*10 + local) incidence list sorted by element (built lazily)
    geo::DevBuf<int32_t> inc_ptr;  // [N+1]
    geo::DevBuf<int32_t> inc;      // [E*10]
    // node-level sparsity pattern (built lazily)
    geo::DevBuf<int64_t> pat_ptr;  // [N+1]
    geo::DevBuf<int32_t> pat_idx;  // [nnz]
    int64_t pat_nnz = -1;
};

struct geo_dofs {
    geo_ctx* ctx = nullptr;
    geo::CtxRef ref;  // declared first after ctx: released after every buffer below
    int64_t n_nodes = 0, n_dofs = 0, n_dir = 0;
    int dpn = 1;
    geo::DevBuf<uint8_t> mask;
    geo::DevBuf<double> vals;
};

struct geo_csr {
    geo_ctx* ctx = nullptr;
    geo::CtxRef ref;  // declared first after ctx: released after every buffer below
    int64_t n_rows = 0, n_cols = 0, nnz = 0;
    geo::DevBuf<int64_t> indptr;
    geo::DevBuf<int32_t> indices;
    geo::DevBuf<double> data;
};

namespace geo {

thread_local inline std::string g_thread_err;

inline void record_error(geo_ctx* ctx, int code, const std::string& msg) {
    (void)code;
    if (ctx) ctx->err = msg;
    g_thread_err = msg;
}

// Checks the launch, then the device error word written by element kernels.
void check_launch(geo_ctx* ctx, const char* what);
// Synchronises the context stream and raises on a CUDA error.
void sync(geo_ctx* ctx, const char* what);
// Clears / reads the context device error word.
void reset_dev_err(geo_ctx* ctx);
int read_dev_err(geo_ctx* ctx);
void raise_dev_err(geo_ctx* ctx, int bits, const char* what);

// Slot `slot` of the context scratch, holding at least n values of T (contents undefined).
template <class T>
T* ctx_scratch(geo_ctx* ctx, int slot, size_t n) {
    ctx->scratch[slot].ensure((n ? n : 1) * sizeof(T));
    return reinterpret_cast<T*>(ctx->scratch[slot].p);
}

// src itself when it is device memory, else a copy in scratch slot `slot` (async on the context stream).
template <class T>
const T* stage_in(geo_ctx* ctx, int slot, const T* src, size_t n) {
    if (n == 0) return nullptr;
    if (is_device_ptr(src)) return src;
    T* d = ctx_scratch<T>(ctx, slot, n);
    GEO_CUDA(cudaMemcpyAsync(d, src, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return d;
}

// assembly.cu
void ensure_inverse_map(geo_mesh* m);
void ensure_pattern(geo_mesh* m);

}  // namespace geo

#define GEO_API_BEGIN(ctxp)                                  \
    geo_ctx* api_ctx_ = (ctxp);                              \
    try {                                                    \
        if (api_ctx_) GEO_CUDA(cudaSetDevice(api_ctx_->device));

#define GEO_API_END                                                                  \
    }                                                                                \
    catch (const geo::Error& e) {                                                    \
        geo::record_error(api_ctx_, e.code, e.msg);                                  \
        return e.code;                                                               \
    }                                                                                \
    catch (const std::bad_alloc&) {                                                  \
        geo::record_error(api_ctx_, GEO_ERR_OUT_OF_MEMORY, "host allocation failed"); \
        return GEO_ERR_OUT_OF_MEMORY;                                                \
    }                                                                                \
    catch (const std::exception& ex) {                                               \
        geo::record_error(api_ctx_, GEO_ERR_INVALID_ARG, ex.what());                 \
        return GEO_ERR_INVALID_ARG;                                                  \
    }                                                                                \
    return GEO_OK;
