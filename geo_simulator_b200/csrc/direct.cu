// Dense LU solve of a CSR system on the device: the drop-in for
// DirectSolver::solve (linalg/direct.rs:28-73), which copies the matrix into a
// dense nalgebra matrix, factors it with partial (row) pivoting and solves.
//
// The matrix is scattered into a dense row-major n x n buffer in HBM (n <=
// kMaxDenseN: 2 GiB). One persistent cooperative kernel then does the whole
// solve, with bounded grid barriers between its phases.
// Factorization, right-looking, two barriers per column k:
//   S. every block combines the per-block pivot candidates of column k (the
//      first row of largest |a_ik|, i >= k: the reference's pivot rule) in the
//      same order, so all blocks agree on the pivot p; rows k and p are swapped
//      (whole rows, as the reference's LU does, and the right-hand side with
//      them), and the multipliers of column k-1, kept aside in lcol, are written
//      below its diagonal;
//   U. rank-1 update of the trailing block and of the right-hand side: each warp
//      owns a row (or a segment of one when there are more warps than rows),
//      forms l_ik = a_ik / a_kk once, skips the row when l_ik == 0 (most rows of
//      a banded FEM matrix), and updates its columns with four 32-wide chunks in
//      flight. The warp owning column k+1 of a row records that row's new
//      a_{i,k+1} as a pivot candidate for the next column, so no separate pivot
//      scan is needed.
// Carrying b through the elimination leaves y = L^-1 P b in place, subtracted
// in the same order as a forward substitution. Back substitution U x = y then
// runs over 32-row blocks from the bottom: every block solves the 32 x 32
// diagonal triangle itself (one warp, identical in all blocks, so no barrier),
// and the grid subtracts its contribution from the rows above, one barrier per
// row block.
// A zero pivot marks the matrix singular (the reference's solve then fails:
// "LU solve failed"); every block sees the same candidates and leaves together.
// ||b - A x|| is formed on the CSR matrix afterwards (solver.rs:139-175).
#include "pcg_common.cuh"

namespace geo {
namespace {

constexpr int kDBS = 256;
constexpr int64_t kMaxDenseN = 16384;

__global__ void k_densify(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                          const double* __restrict__ data, int64_t n, double* __restrict__ M) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) M[i * n + indices[p]] = data[p];
}

struct LuArgs {
    double* M;
    int64_t n;
    double* y;          // in: b; after the elimination L^-1 P b
    double* x;          // out: the solution
    double* lcol;       // multipliers of the last eliminated column, by row
    double* cand_val;   // per-block pivot candidate (signed value)
    int64_t* cand_idx;  // its row, n when the block has none
    int* singular;
    GridSync* gs;
    unsigned long long timeout_ns;
};

// Keeps (v, i) when |v| is larger, or equal with a smaller row: the first maximum.
__device__ __forceinline__ void cand_merge(double& bv, int64_t& bi, double v, int64_t i) {
    if (fabs(v) > fabs(bv) || (fabs(v) == fabs(bv) && i < bi)) {
        bv = v;
        bi = i;
    }
}

// Block-wide first maximum of the threads' candidates -> cand_*[blockIdx.x].
__device__ void store_candidate(const LuArgs& a, double bv, int64_t bi) {
    __shared__ double s_val[kDBS / 32];
    __shared__ int64_t s_idx[kDBS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, bv, o);
        const int64_t oi = __shfl_down_sync(0xffffffffu, bi, o);
        cand_merge(bv, bi, ov, oi);
    }
    if ((threadIdx.x & 31) == 0) {
        s_val[threadIdx.x >> 5] = bv;
        s_idx[threadIdx.x >> 5] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kDBS / 32; ++w) cand_merge(s_val[0], s_idx[0], s_val[w], s_idx[w]);
        __stcg(a.cand_val + blockIdx.x, s_val[0]);
        __stcg(a.cand_idx + blockIdx.x, s_idx[0]);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kDBS) k_lu(LuArgs a) {
    __shared__ double s_piv_val;
    __shared__ int64_t s_piv;
    const int64_t n = a.n;
    const int lane = threadIdx.x & 31;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t gw = tid >> 5, nw = nth >> 5;
    {  // candidates of column 0; rows visited in increasing order keep the first maximum
        double bv = 0.0;
        int64_t bi = n;
        for (int64_t i = tid; i < n; i += nth) {
            const double v = a.M[i * n];
            if (bi == n || fabs(v) > fabs(bv)) {
                bv = v;
                bi = i;
            }
        }
        store_candidate(a, bv, bi);
    }
    if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;
    for (int64_t k = 0; k < n; ++k) {
        // ---- S: pivot, swap, multipliers of column k-1
        if (threadIdx.x < 32) {
            double bv = 0.0;
            int64_t bi = n;
            for (unsigned b = lane; b < gridDim.x; b += 32) {
                const int64_t ci = __ldcg(a.cand_idx + b);
                if (ci < n) cand_merge(bv, bi, __ldcg(a.cand_val + b), ci);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, bv, o);
                const int64_t oi = __shfl_down_sync(0xffffffffu, bi, o);
                cand_merge(bv, bi, ov, oi);
            }
            if (lane == 0) {
                s_piv_val = bv;
                s_piv = (bi < n && bv != 0.0) ? bi : -1;
            }
        }
        __syncthreads();
        const int64_t p = s_piv;
        const double d = s_piv_val;
        if (p < 0) {  // every block reads the same candidates: all leave here
            if (tid == 0) *a.singular = 1;
            return;
        }
        if (k > 0)
            for (int64_t i = k + tid; i < n; i += nth) {
                const int64_t src = i == k ? p : (i == p ? k : i);
                a.M[i * n + k - 1] = a.lcol[src];
            }
        if (p != k) {
            for (int64_t j = tid; j < n; j += nth) {
                if (j == k - 1) continue;
                const double t = a.M[k * n + j];
                a.M[k * n + j] = a.M[p * n + j];
                a.M[p * n + j] = t;
            }
            if (tid == 0) {
                const double t = a.y[k];
                a.y[k] = a.y[p];
                a.y[p] = t;
            }
        }
        const int64_t m = n - k - 1;
        if (m == 0) break;
        if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;
        // ---- U: trailing update, candidates of column k+1
        const int64_t nch = (m + 31) / 32;  // 32-column chunks of columns k+1..n-1
        const int64_t W = m >= nw ? 1 : std::min<int64_t>(nch, nw / m);
        const double* pk = a.M + k * n;
        const double yk = a.y[k];
        double bv = 0.0;
        int64_t bi = n;
        for (int64_t t = gw; t < m * W; t += nw) {
            const int64_t i = k + 1 + t / W, s = t % W;
            double* pi = a.M + i * n;
            const double l = pi[k] / d;
            if (s == 0 && lane == 0) {
                a.lcol[i] = l;
                if (l != 0.0) a.y[i] -= l * yk;
            }
            if (l != 0.0) {
                const int64_t jb = k + 1 + (s * nch / W) * 32;
                const int64_t je = std::min<int64_t>(n, k + 1 + ((s + 1) * nch / W) * 32);
                for (int64_t j = jb + lane; j < je; j += 128) {
                    double ai[4], ak[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int64_t jj = j + 32 * u;
                        ai[u] = jj < je ? pi[jj] : 0.0;
                        ak[u] = jj < je ? pk[jj] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (j + 32 * u < je) pi[j + 32 * u] = ai[u] - l * ak[u];
                }
            }
            if (s == 0 && lane == 0) {  // this lane wrote (or left) a_{i,k+1}
                const double v = pi[k + 1];
                if (bi == n || fabs(v) > fabs(bv)) {
                    bv = v;
                    bi = i;
                }
            }
        }
        store_candidate(a, bv, bi);
        if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;
    }
    // ---- back substitution U x = y over 32-row blocks, bottom first
    __shared__ double s_x[32];
    if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;  // the last swap of y
    for (int64_t r0 = (n - 1) / 32 * 32; r0 >= 0; r0 -= 32) {
        const int64_t r1 = std::min<int64_t>(n, r0 + 32);
        if (threadIdx.x < 32) {  // the diagonal triangle, the same in every block
            const int64_t j = r0 + lane;
            double xj = 0.0;
            for (int64_t r = r1 - 1; r >= r0; --r) {
                double t = (j > r && j < r1) ? a.M[r * n + j] * xj : 0.0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
                t = __shfl_sync(0xffffffffu, t, 0);
                if (j == r) xj = (a.y[r] - t) / a.M[r * n + r];
            }
            s_x[lane] = xj;
            if (blockIdx.x == 0 && j < r1) a.x[j] = xj;
        }
        __syncthreads();
        if (r0 == 0) break;
        for (int64_t i = gw; i < r0; i += nw) {  // rows above: y_i -= U[i, r0:r1] x[r0:r1]
            const int64_t j = r0 + lane;
            double t = j < r1 ? a.M[i * n + j] * s_x[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) a.y[i] -= t;
        }
        if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;
    }
}

// Per-block partials of ||b - A x||^2 and ||b||^2 (CSR)
__global__ void __launch_bounds__(kDBS) k_residual(const int64_t* __restrict__ indptr,
                                                   const int32_t* __restrict__ indices,
                                                   const double* __restrict__ data, int64_t n,
                                                   const double* __restrict__ x, const double* __restrict__ b,
                                                   double* __restrict__ part) {
    double v[2] = {0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double ax = 0.0;
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) ax += data[p] * x[indices[p]];
        const double r = b[i] - ax;
        v[0] += r * r;
        v[1] += b[i] * b[i];
    }
    store_partial<2>(part, v);
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

int geo_direct_solve(geo_ctx* ctx, const geo_csr* A, const double* b, double* x, geo_solver_stats* stats) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && A && b && x, "NULL argument");
    GEO_CHECK_ARG(A->n_rows == A->n_cols, "matrix must be square");
    const int64_t n = A->n_rows;
    GEO_CHECK_ARG(n >= 1 && n <= kMaxDenseN, "dense LU: n must be in 1..16384 (n x n doubles on the device)");
    cudaStream_t s = ctx->stream;
    DevBuf<double> tb, M((size_t)n * n), vec(3 * (size_t)n);
    const double* db = stage_in(b, (size_t)n, tb, s);
    double *lcol = vec.p, *y = vec.p + n, *xd = vec.p + 2 * n;
    GEO_CUDA(cudaMemcpyAsync(y, db, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const int nb = (int)std::max<int64_t>(
        1, std::min<int64_t>(persistent_blocks(ctx, k_lu, kDBS, 0), cdiv(n * n, 4 * kDBS)));
    DevBuf<double> cv(nb);
    DevBuf<int64_t> ci(nb);
    DevBuf<int> sing(1);
    DevBuf<GridSync> gs(1);
    GEO_CUDA(cudaMemsetAsync(M.p, 0, M.bytes(), s));
    GEO_CUDA(cudaMemsetAsync(gs.p, 0, sizeof(GridSync), s));
    GEO_CUDA(cudaMemsetAsync(sing.p, 0, sizeof(int), s));
    GEO_CUDA(cudaEventRecord(ctx->ev0, s));
    k_densify<<<(unsigned)std::min<int64_t>(cdiv(n, kDBS), 4096), kDBS, 0, s>>>(A->indptr.p, A->indices.p,
                                                                               A->data.p, n, M.p);
    check_launch(ctx, "k_densify");
    LuArgs la{M.p, n, y, xd, lcol, cv.p, ci.p, sing.p, gs.p, 10ull * 1000000000ull};
    launch_persistent(ctx, k_lu, kDBS, 0, la, nb);
    GEO_CUDA(cudaEventRecord(ctx->ev1, s));
    int singular = 0;
    GridSync g{};
    GEO_CUDA(cudaMemcpyAsync(&singular, sing.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GEO_CUDA(cudaMemcpyAsync(&g, gs.p, sizeof(g), cudaMemcpyDeviceToHost, s));
    sync(ctx, "dense LU");
    if (g.error & DEV_ERR_TIMEOUT) fail(GEO_ERR_TIMEOUT, "dense LU: grid barrier timed out");
    if (singular) fail(GEO_ERR_SINGULAR_MATRIX, "LU solve failed: the matrix is singular");
    const int rb = (int)std::min<int64_t>(cdiv(n, kDBS), 1024);
    DevBuf<double> part((size_t)rb * 2);
    k_residual<<<rb, kDBS, 0, s>>>(A->indptr.p, A->indices.p, A->data.p, n, xd, db, part.p);
    check_launch(ctx, "k_residual");
    std::vector<double> hp((size_t)rb * 2);
    GEO_CUDA(cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    copy_out(x, xd, (size_t)n, s);
    sync(ctx, "geo_direct_solve");
    double rr = 0.0, bb = 0.0;
    for (int i = 0; i < rb; ++i) {
        rr += hp[2 * (size_t)i];
        bb += hp[2 * (size_t)i + 1];
    }
    float ms = 0.f;
    GEO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    const double res = std::sqrt(rr), bn = std::sqrt(bb);
    const double rel = bn < 1e-14 ? res : res / bn;  // solver.rs:165-175
    if (stats) {
        *stats = geo_solver_stats{};
        stats->iterations = 0;  // direct.rs:62
        stats->residual_norm = res;
        stats->relative_residual = rel;
        stats->converged = rel < 1e-8;  // direct.rs:65
        stats->solve_time = ms * 1e-3;
        stats->kernel_time = ms * 1e-3;
        stats->status = GEO_OK;
        stats->b_norm = bn;
        stats->kernel_launches = 3;
    }
    GEO_API_END
}

}  // extern "C"
