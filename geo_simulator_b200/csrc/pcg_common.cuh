// Shared pieces of the persistent PCG kernels (CSR and matrix-free).
#pragma once

#include <algorithm>

#include "objects.h"

namespace geo {

// Written by block 0 of a persistent solve.
struct PcgResult {
    long long iterations;
    double residual_norm;
    double b_norm;
    int converged;
    int breakdown;
    long long fp64_updates;
};

inline void cg_opts_fill(const geo_cg_opts* in, geo_cg_opts& o) {
    geo_cg_opts_default(&o);
    if (in) o = *in;
    if (o.timeout_seconds <= 0) o.timeout_seconds = 10.0;
    if (o.reliable_delta <= 0 || o.reliable_delta >= 1) o.reliable_delta = 0.1;
}

// Workspace owned by the persistent kernels: barrier word, result, partials.
struct PcgScratch {
    DevBuf<GridSync> gs;
    DevBuf<PcgResult> res;
    DevBuf<double> part;  // [3 slots][nblocks][4]
    void ensure(int nblocks) {
        if (!gs.p) gs.alloc(1);
        if (!res.p) res.alloc(1);
        part.ensure((size_t)3 * nblocks * 4);
    }
    double* slot(int k, int nblocks) { return part.p + (size_t)k * nblocks * 4; }
};

// Launches a co-resident persistent grid (cooperative launch) of `bs` threads,
// sized by the occupancy calculator; returns the number of blocks used.
template <class Kernel, class Args>
int launch_persistent(geo_ctx* ctx, Kernel kernel, int bs, size_t smem, Args& args, int nblocks) {
    void* params[] = {&args};
    GEO_CUDA(cudaLaunchCooperativeKernel((const void*)kernel, dim3(nblocks), dim3(bs), params, smem,
                                         ctx->stream));
    return nblocks;
}

template <class Kernel>
int persistent_blocks(geo_ctx* ctx, Kernel kernel, int bs, size_t smem) {
    int per_sm = 0;
    GEO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, bs, smem));
    if (per_sm < 1) fail(GEO_ERR_UNSUPPORTED, "persistent kernel does not fit on an SM");
    return per_sm * ctx->sm_count;
}

inline void fill_stats(geo_solver_stats* st, const PcgResult& r, double seconds, int status) {
    if (!st) return;
    st->iterations = r.iterations;
    st->residual_norm = r.residual_norm;
    st->relative_residual = r.b_norm > 1e-20 ? r.residual_norm / r.b_norm : 0.0;
    st->converged = r.converged;
    st->solve_time = seconds;
    st->status = status;
    st->fp64_residual_updates = r.fp64_updates;
    st->b_norm = r.b_norm;
    st->kernel_time = seconds;
}

}  // namespace geo
