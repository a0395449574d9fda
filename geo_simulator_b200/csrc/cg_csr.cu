// K4: FP64 Jacobi-PCG on an assembled CSR matrix, the drop-in for
// ConjugateGradient::solve (linalg/iterative.rs:46-131) with
// JacobiPreconditioner (linalg/preconditioner.rs:37-62).
//
// One persistent cooperative kernel runs the whole solve: sub-warp SpMV,
// Jacobi scaling, axpys, and dot products reduced by warp shuffles into
// per-block partials that every block sums in the same fixed order after a
// bounded grid barrier (so all blocks take identical, deterministic decisions).
#include <mutex>

#include "pcg_common.cuh"

namespace geo {
namespace {

constexpr int kBS = 256;
#ifndef GEO_CSR_VEC
#define GEO_CSR_VEC 4
#endif
#ifndef GEO_CSR_UNROLL
#define GEO_CSR_UNROLL 8
#endif
// The SpMV is bound by load latency: each row group takes two dependent round trips
// (values and indices, then the gathers of p). Four lanes per row with eight entries
// each covers a Tet10 row (about 28 entries) in one step and puts eight rows per
// warp in flight: 0.230 ms per PCG iteration at 64^3 (59.8M entries), against 0.274
// ms with eight lanes x four entries and 0.239 ms with two lanes x sixteen.
constexpr int kVec = GEO_CSR_VEC;           // lanes per CSR row
constexpr int kUnrollCsr = GEO_CSR_UNROLL;  // row entries in flight per lane in the SpMV

struct CsrPcgArgs {
    const int64_t* indptr;
    const int32_t* indices;
    const double* data;
    int64_t n;
    const double* b;
    double *x, *r, *p, *q, *dinv;
    double *part_a, *part_b;
    GridSync* gs;
    PcgResult* res;
    unsigned long long timeout_ns;
    long long max_it;
    double tol, abs_tol;
    int use_prec;
};

__device__ __forceinline__ int64_t lower_bound_i32(const int32_t* idx, int64_t b, int64_t e, int32_t c) {
    while (b < e) {
        const int64_t m = (b + e) >> 1;
        if (idx[m] < c) b = m + 1;
        else e = m;
    }
    return b;
}

__global__ void __launch_bounds__(kBS, 4) k_csr_pcg(CsrPcgArgs a) {
    const unsigned nb = gridDim.x;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t n = a.n;

    // x = 0, r = b, z = M^-1 r, p = z (iterative.rs:70-75)
    {
        double v[2] = {0.0, 0.0};
        for (int64_t i = tid; i < n; i += nth) {
            double di = 1.0;
            if (a.use_prec) {
                const int64_t rb = a.indptr[i], re = a.indptr[i + 1];
                const int64_t pp = lower_bound_i32(a.indices, rb, re, (int32_t)i);
                if (pp < re && a.indices[pp] == i) {
                    const double d = a.data[pp];
                    if (fabs(d) > 1e-14) di = 1.0 / d;
                }
            }
            a.dinv[i] = di;
            const double bi = a.b[i];
            const double zi = bi * di;
            a.x[i] = 0.0;
            a.r[i] = bi;
            a.p[i] = zi;
            v[0] += bi * bi;
            v[1] += bi * zi;
        }
        store_partial<2>(a.part_b, v);
    }
    if (!grid_barrier(a.gs, nb, a.timeout_ns)) return;
    double t2[2];
    grid_total<2>(a.part_b, nb, t2);
    const double bnorm = sqrt(t2[0]);
    double rz = t2[1];
    if (bnorm < 1e-25) {  // iterative.rs:60-68
        if (tid == 0) *a.res = PcgResult{0, 0.0, bnorm, 1, 0, 0};
        return;
    }
    long long it = 0;
    int converged = 0, breakdown = 0;
    double final_res = bnorm;
    const int lane = threadIdx.x & 31, sub = lane % kVec;
    const int64_t warp = tid >> 5, nwarps = nth >> 5;
    constexpr int rows_per_warp = 32 / kVec;
    while (it < a.max_it) {
        // q = A p and p.q
        {
            double v[1] = {0.0};
            for (int64_t rbase = warp * rows_per_warp; rbase < n; rbase += nwarps * rows_per_warp) {
                const int64_t row = rbase + lane / kVec;
                double s = 0.0;
                if (row < n) {
                    // kUnroll entries per lane in flight: all value/index loads, then all
                    // gathers of p, then the products in the original order (same sum)
                    const int64_t re = __ldg(a.indptr + row + 1);
                    for (int64_t pp0 = __ldg(a.indptr + row) + sub; pp0 < re; pp0 += kUnrollCsr * kVec) {
                        double d[kUnrollCsr], pv[kUnrollCsr];
                        int32_t c[kUnrollCsr];
#pragma unroll
                        for (int u = 0; u < kUnrollCsr; ++u) {
                            const int64_t pp = pp0 + (int64_t)u * kVec;
                            d[u] = pp < re ? __ldg(a.data + pp) : 0.0;
                            c[u] = pp < re ? __ldg(a.indices + pp) : -1;
                        }
#pragma unroll
                        for (int u = 0; u < kUnrollCsr; ++u) pv[u] = c[u] >= 0 ? a.p[c[u]] : 0.0;
#pragma unroll
                        for (int u = 0; u < kUnrollCsr; ++u)
                            if (c[u] >= 0) s += d[u] * pv[u];
                    }
                }
#pragma unroll
                for (int o = kVec / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, kVec);
                if (row < n && sub == 0) {
                    a.q[row] = s;
                    v[0] += a.p[row] * s;
                }
            }
            store_partial<1>(a.part_a, v);
        }
        if (!grid_barrier(a.gs, nb, a.timeout_ns)) return;
        double pq[1];
        grid_total<1>(a.part_a, nb, pq);
        if (fabs(pq[0]) < 1e-30) {  // iterative.rs:85
            breakdown = 1;
            break;
        }
        const double alpha = rz / pq[0];
        {
            double v[2] = {0.0, 0.0};
            for (int64_t i = tid; i < n; i += nth) {
                const double pi = a.p[i];
                a.x[i] += alpha * pi;
                const double ri = a.r[i] - alpha * a.q[i];
                a.r[i] = ri;
                v[0] += ri * ri;
                v[1] += ri * (ri * a.dinv[i]);
            }
            store_partial<2>(a.part_b, v);
        }
        if (!grid_barrier(a.gs, nb, a.timeout_ns)) return;
        grid_total<2>(a.part_b, nb, t2);
        const double rn = sqrt(t2[0]);
        final_res = rn;
        if (rn < a.tol * bnorm || rn < a.abs_tol) {  // iterative.rs:95
            converged = 1;
            break;
        }
        const double beta = t2[1] / rz;
        rz = t2[1];
        for (int64_t i = tid; i < n; i += nth) a.p[i] = a.r[i] * a.dinv[i] + beta * a.p[i];
        if (!grid_barrier(a.gs, nb, a.timeout_ns)) return;
        ++it;
    }
    if (tid == 0) *a.res = PcgResult{it, final_res, bnorm, converged, breakdown, 0};
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

void geo_cg_opts_default(geo_cg_opts* o) {
    if (!o) return;
    o->max_iterations = 1000;
    o->tolerance = 1e-8;
    o->abs_tolerance = 1e-12;
    o->use_preconditioner = 1;
    o->precision = GEO_PRECISION_FP64;
    o->reliable_delta = 0.1;
    o->timeout_seconds = 10.0;
}

int geo_cg_solve(geo_ctx* ctx, const geo_csr* A, const double* b, const geo_cg_opts* opts, double* x,
                 geo_solver_stats* stats) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && A && b && x, "NULL argument");
    GEO_CHECK_ARG(A->n_rows == A->n_cols, "matrix must be square");
    geo_cg_opts o;
    cg_opts_fill(opts, o);
    GEO_CHECK_ARG(o.max_iterations >= 0, "max_iterations must be >= 0");
    cudaStream_t s = ctx->stream;
    const int64_t n = A->n_rows;
    DevBuf<double> tb, work(5 * n);
    const double* db = stage_in(b, n, tb, s);
    const int nb = persistent_blocks(ctx, k_csr_pcg, kBS, 0);
    PcgScratch sc;
    sc.ensure(nb);
    CsrPcgArgs args{};
    args.indptr = A->indptr.p;
    args.indices = A->indices.p;
    args.data = A->data.p;
    args.n = n;
    args.b = db;
    args.x = work.p;
    args.r = work.p + n;
    args.p = work.p + 2 * n;
    args.q = work.p + 3 * n;
    args.dinv = work.p + 4 * n;
    args.part_a = sc.slot(0, nb);
    args.part_b = sc.slot(1, nb);
    args.gs = sc.gs.p;
    args.res = sc.res.p;
    args.timeout_ns = (unsigned long long)(o.timeout_seconds * 1e9);
    args.max_it = o.max_iterations;
    args.tol = o.tolerance;
    args.abs_tol = o.abs_tolerance;
    args.use_prec = o.use_preconditioner;
    GEO_CUDA(cudaMemsetAsync(sc.gs.p, 0, sizeof(GridSync), s));
    GEO_CUDA(cudaMemsetAsync(sc.res.p, 0, sizeof(PcgResult), s));
    GEO_CUDA(cudaEventRecord(ctx->ev0, s));
    launch_persistent(ctx, k_csr_pcg, kBS, 0, args, nb);
    GEO_CUDA(cudaEventRecord(ctx->ev1, s));
    PcgResult r{};
    GridSync g{};
    GEO_CUDA(cudaMemcpyAsync(&r, sc.res.p, sizeof(r), cudaMemcpyDeviceToHost, s));
    GEO_CUDA(cudaMemcpyAsync(&g, sc.gs.p, sizeof(g), cudaMemcpyDeviceToHost, s));
    copy_out(x, work.p, n, s);
    sync(ctx, "geo_cg_solve");
    float ms = 0.f;
    GEO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (g.error & DEV_ERR_TIMEOUT) {
        fill_stats(stats, r, ms * 1e-3, GEO_ERR_TIMEOUT);
        fail(GEO_ERR_TIMEOUT, "PCG grid barrier timed out");
    }
    const int status = r.converged ? GEO_OK : (r.breakdown ? GEO_ERR_BREAKDOWN : GEO_NOT_CONVERGED);
    fill_stats(stats, r, ms * 1e-3, status);
    if (stats) stats->kernel_launches = 1;
    if (status != GEO_OK) {
        record_error(ctx, status, r.breakdown ? "CG breakdown: |p^T A p| < 1e-30" : "CG did not converge");
        return status;
    }
    GEO_API_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of geo_cg_solve (no counterpart in the reference).
//
// Who needs it: callers that must not call cudaMalloc/cudaFree between solves --
// a host loop whose device memory is fully reserved by another allocator (a
// caching allocator that has already taken the free memory), or a latency loop
// that cannot afford cudaFree's implicit device-wide synchronisation. It runs the
// same k_csr_pcg kernel as geo_cg_solve, with the four work vectors, the block
// partials, the barrier word and the result taken from one file-scope device
// array instead of cudaMalloc, so results are bit-identical to geo_cg_solve.
//
// Limits and rules:
//  * at most GEO_NOALLOC_MAX_ROWS rows and kNoAllocMaxBlocks persistent blocks;
//    larger systems are rejected with GEO_ERR_INVALID_ARG;
//  * b and x must be device memory on the context's device (no host staging);
//  * the GridSync word and the PcgResult slot must start at zero: they are
//    cleared with cudaMemsetAsync on the context stream before every launch
//    (a timed-out barrier can leave the count non-zero);
//  * one scratch array per device: two calls that overlap on the same device
//    (different threads or contexts) race on it and must be serialised;
//  * the first call on a device looks the array up with cudaGetSymbolAddress,
//    which can make the runtime load this module and reserve the array; make
//    that first call before the phase that must not allocate, and before any
//    stream capture begins. The address is kept per device together with the
//    driver's unique id of the device's current context; after a
//    cudaDeviceReset the context (and its id) is new, so the next call looks the
//    array up again instead of using an address of the old context.
namespace geo {
namespace {

constexpr int kNoAllocMaxBlocks = 4096;
constexpr size_t kNoAllocVecBytes = (size_t)GEO_NOALLOC_MAX_ROWS * sizeof(double);
constexpr size_t kNoAllocPartBytes = (size_t)kNoAllocMaxBlocks * 4 * sizeof(double);
constexpr size_t kNoAllocOffPart = 4 * kNoAllocVecBytes;                    // r, p, q, dinv
constexpr size_t kNoAllocOffSync = kNoAllocOffPart + 2 * kNoAllocPartBytes;  // part_a, part_b
constexpr size_t kNoAllocOffRes = kNoAllocOffSync + 256;
constexpr size_t kNoAllocBytes = kNoAllocOffRes + 256;
static_assert(sizeof(GridSync) <= 256 && sizeof(PcgResult) <= 256, "scratch slots too small");
static_assert(kNoAllocVecBytes % 256 == 0 && kNoAllocPartBytes % 256 == 0, "slots stay 256-byte aligned");

// 8.25 MiB per device: 4 x 2 MiB vectors + 2 x 128 KiB partials + two 256 B slots.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {};
unsigned long long g_noalloc_ctx_id[kNoAllocMaxDevices] = {};

// Unique id of the calling thread's current driver context (cuCtxGetId through
// the runtime's driver entry point, so the library needs no -lcuda); 0 when the
// driver cannot say, in which case the cached address is trusted as before.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    void* c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == 0 && c && get_id(c, &id) == 0) return id;
    return 0;
}

// Device address of g_noalloc_scratch on `device` (which must be current),
// looked up once per device and context.
unsigned char* noalloc_scratch(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices) fail(GEO_ERR_UNSUPPORTED, "device ordinal out of range");
    const unsigned long long ctx_id = current_context_id();
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device] || g_noalloc_ctx_id[device] != ctx_id) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            fail(GEO_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[device] = static_cast<unsigned char*>(p);
        g_noalloc_ctx_id[device] = ctx_id;
    }
    return g_noalloc_addr[device];
}

bool on_device(const void* p, int device) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

}  // namespace
}  // namespace geo

extern "C" int geo_cg_solve_noalloc(geo_ctx* ctx, const geo_csr* A, const double* b_dev,
                                    const geo_cg_opts* opts, double* x_dev, geo_solver_stats* stats) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && A, "NULL argument");
    unsigned char* base = noalloc_scratch(ctx->device);  // first call: symbol lookup
    GEO_CHECK_ARG(A->n_rows == A->n_cols, "matrix must be square");
    const int64_t n = A->n_rows;
    if (n > GEO_NOALLOC_MAX_ROWS)
        fail(GEO_ERR_INVALID_ARG, "geo_cg_solve_noalloc: " + std::to_string(n) +
                                      " rows exceed GEO_NOALLOC_MAX_ROWS (" +
                                      std::to_string((long long)GEO_NOALLOC_MAX_ROWS) + "); use geo_cg_solve");
    if (n > 0)
        GEO_CHECK_ARG(b_dev && x_dev && on_device(b_dev, ctx->device) && on_device(x_dev, ctx->device),
                      "geo_cg_solve_noalloc: b and x must be device memory on the context's device");
    geo_cg_opts o;
    cg_opts_fill(opts, o);
    GEO_CHECK_ARG(o.max_iterations >= 0, "max_iterations must be >= 0");
    const int nb = persistent_blocks(ctx, k_csr_pcg, kBS, 0);
    if (nb > kNoAllocMaxBlocks) fail(GEO_ERR_UNSUPPORTED, "geo_cg_solve_noalloc: persistent grid too large");
    cudaStream_t s = ctx->stream;
    double* vec = reinterpret_cast<double*>(base);
    GridSync* gs = reinterpret_cast<GridSync*>(base + kNoAllocOffSync);
    PcgResult* res = reinterpret_cast<PcgResult*>(base + kNoAllocOffRes);
    CsrPcgArgs args{};
    args.indptr = A->indptr.p;
    args.indices = A->indices.p;
    args.data = A->data.p;
    args.n = n;
    args.b = b_dev;
    args.x = x_dev;
    args.r = vec;
    args.p = vec + GEO_NOALLOC_MAX_ROWS;
    args.q = vec + 2 * (size_t)GEO_NOALLOC_MAX_ROWS;
    args.dinv = vec + 3 * (size_t)GEO_NOALLOC_MAX_ROWS;
    args.part_a = reinterpret_cast<double*>(base + kNoAllocOffPart);
    args.part_b = reinterpret_cast<double*>(base + kNoAllocOffPart + kNoAllocPartBytes);
    args.gs = gs;
    args.res = res;
    args.timeout_ns = (unsigned long long)(o.timeout_seconds * 1e9);
    args.max_it = o.max_iterations;
    args.tol = o.tolerance;
    args.abs_tol = o.abs_tolerance;
    args.use_prec = o.use_preconditioner;
    GEO_CUDA(cudaMemsetAsync(gs, 0, sizeof(GridSync), s));
    GEO_CUDA(cudaMemsetAsync(res, 0, sizeof(PcgResult), s));
    GEO_CUDA(cudaEventRecord(ctx->ev0, s));
    launch_persistent(ctx, k_csr_pcg, kBS, 0, args, nb);
    GEO_CUDA(cudaEventRecord(ctx->ev1, s));
    PcgResult r{};
    GridSync g{};
    GEO_CUDA(cudaMemcpyAsync(&r, res, sizeof(r), cudaMemcpyDeviceToHost, s));
    GEO_CUDA(cudaMemcpyAsync(&g, gs, sizeof(g), cudaMemcpyDeviceToHost, s));
    sync(ctx, "geo_cg_solve_noalloc");
    float ms = 0.f;
    GEO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (g.error & DEV_ERR_TIMEOUT) {
        fill_stats(stats, r, ms * 1e-3, GEO_ERR_TIMEOUT);
        fail(GEO_ERR_TIMEOUT, "PCG grid barrier timed out");
    }
    const int status = r.converged ? GEO_OK : (r.breakdown ? GEO_ERR_BREAKDOWN : GEO_NOT_CONVERGED);
    fill_stats(stats, r, ms * 1e-3, status);
    if (stats) stats->kernel_launches = 1;
    if (status != GEO_OK) {
        record_error(ctx, status, r.breakdown ? "CG breakdown: |p^T A p| < 1e-30" : "CG did not converge");
        return status;
    }
    GEO_API_END
}
