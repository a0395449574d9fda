// BiCGSTAB and restarted GMRES on an assembled CSR matrix, FP64: the drop-ins for
// BiCGSTAB::solve (linalg/iterative.rs:150-301) and GMRES::solve (:303-479), the
// siblings of ConjugateGradient in the reference's iterative-solver file. Both
// are right-preconditioned with the Jacobi inverse diagonal
// (linalg/preconditioner.rs:37-62) or the identity, and keep the reference's
// stopping rules, breakdown thresholds and iteration counting.
//
// Each solve is one persistent cooperative kernel, as the CG drop-in: sub-warp
// CSR SpMV with several row entries in flight per lane, element-wise passes, and
// dot products reduced to per-block partials that every block sums in the same
// fixed order after a bounded grid barrier, so all blocks take the same
// decisions. Partials alternate between two buffers by a running count, so a
// block can store the next partials while a slower one still reads the last.
// GMRES keeps the Hessenberg matrix, the Givens rotations and the rotated
// right-hand side in shared memory in every block (computed identically from
// the reduced values), and its Krylov basis ((restart + 1) x n) in HBM.
#include "pcg_common.cuh"

namespace geo {
namespace {

constexpr int kKBS = 256;
// SpMV row shape (lanes per CSR row, row entries in flight per lane): GMRES takes
// the CG drop-in's four lanes x eight entries; BiCGSTAB, with two SpMVs and more
// live vectors, keeps eight x four, which fits its 64 registers without spills.
constexpr int kGmresVec = 4, kGmresUnroll = 8;
constexpr int kBicgVec = 8, kBicgUnroll = 4;
constexpr int kMaxRestart = 64;

struct KrylovArgs {
    const int64_t* indptr;
    const int32_t* indices;
    const double* data;
    int64_t n;
    const double* b;
    double* x;
    double* dinv;
    double* w[8];  // work vectors
    double* V;     // GMRES basis, (restart + 1) x n
    double* part[2];
    GridSync* gs;
    PcgResult* res;
    unsigned long long timeout_ns;
    long long max_it;
    int restart;
    double tol, abs_tol;
    int use_prec;
};

// (A x)_row for the sub-warp of kKVec lanes owning `row` (valid in lane sub == 0)
template <int kKVec, int kKUnroll>
__device__ __forceinline__ double csr_row(const KrylovArgs& a, int64_t row, int sub, const double* x) {
    double s = 0.0;
    if (row < a.n) {
        const int64_t re = __ldg(a.indptr + row + 1);
        for (int64_t pp0 = __ldg(a.indptr + row) + sub; pp0 < re; pp0 += kKUnroll * kKVec) {
            double d[kKUnroll], xv[kKUnroll];
            int32_t c[kKUnroll];
#pragma unroll
            for (int u = 0; u < kKUnroll; ++u) {
                const int64_t pp = pp0 + (int64_t)u * kKVec;
                d[u] = pp < re ? __ldg(a.data + pp) : 0.0;
                c[u] = pp < re ? __ldg(a.indices + pp) : -1;
            }
#pragma unroll
            for (int u = 0; u < kKUnroll; ++u) xv[u] = c[u] >= 0 ? x[c[u]] : 0.0;
#pragma unroll
            for (int u = 0; u < kKUnroll; ++u)
                if (c[u] >= 0) s += d[u] * xv[u];
        }
    }
#pragma unroll
    for (int o = kKVec / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, kKVec);
    return s;
}

// Jacobi inverse diagonal (1/A_ii if |A_ii| > 1e-14, else 1) or the identity
__device__ void init_dinv(const KrylovArgs& a, int64_t tid, int64_t nth) {
    for (int64_t i = tid; i < a.n; i += nth) {
        double di = 1.0;
        if (a.use_prec) {
            int64_t lo = a.indptr[i], hi = a.indptr[i + 1];
            const int64_t re = hi;
            while (lo < hi) {
                const int64_t m = (lo + hi) >> 1;
                if (a.indices[m] < (int32_t)i) lo = m + 1;
                else hi = m;
            }
            if (lo < re && a.indices[lo] == i) {
                const double d = a.data[lo];
                if (fabs(d) > 1e-14) di = 1.0 / d;
            }
        }
        a.dinv[i] = di;
    }
}

// Grid reduction of K per-thread values: partials into the buffer of turn t, barrier, totals.
template <int K>
__device__ __forceinline__ bool reduce(const KrylovArgs& a, int& turn, double (&v)[K], double (&out)[K]) {
    double* part = a.part[turn & 1];
    ++turn;
    store_partial<K>(part, v);
    if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return false;
    grid_total<K>(part, gridDim.x, out);
    return true;
}

// ------------------------------------------------------------------ BiCGSTAB (iterative.rs:177-278)
__global__ void __launch_bounds__(kKBS, 4) k_bicgstab(KrylovArgs a) {
    constexpr int kKVec = kBicgVec;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31, sub = lane % kKVec;
    const int64_t warp = tid >> 5, nwarps = nth >> 5;
    constexpr int rows_per_warp = 32 / kKVec;
    const int64_t n = a.n;
    double *r = a.w[0], *rh = a.w[1], *p = a.w[2], *v = a.w[3], *s = a.w[4], *t = a.w[5], *ph = a.w[6],
           *sh = a.w[7];
    int turn = 0;
    init_dinv(a, tid, nth);
    double bnorm;
    {
        double q[1] = {0.0}, o[1];
        for (int64_t i = tid; i < n; i += nth) {
            const double bi = a.b[i];
            a.x[i] = 0.0;
            r[i] = bi;
            rh[i] = bi;
            v[i] = 0.0;
            p[i] = 0.0;
            q[0] += bi * bi;
        }
        if (!reduce<1>(a, turn, q, o)) return;
        bnorm = sqrt(o[0]);
    }
    if (bnorm < 1e-25) {
        if (tid == 0) *a.res = PcgResult{0, 0.0, bnorm, 1, 0, 0};
        return;
    }
    double rho = 1.0, alpha = 1.0, omega = 1.0, final_res = bnorm;
    long long it = 0;
    int converged = 0, breakdown = 0;
    while (it < a.max_it) {
        const double rho_prev = rho;
        {
            double q[1] = {0.0}, o[1];
            for (int64_t i = tid; i < n; i += nth) q[0] += rh[i] * r[i];
            if (!reduce<1>(a, turn, q, o)) return;
            rho = o[0];
        }
        if (fabs(rho) < 1e-40) {
            breakdown = 1;
            break;
        }
        const double beta = it == 0 ? 0.0 : (rho / rho_prev) * (alpha / omega);
        for (int64_t i = tid; i < n; i += nth) {
            const double pi = it == 0 ? r[i] : r[i] + beta * (p[i] - omega * v[i]);
            p[i] = pi;
            ph[i] = pi * a.dinv[i];
        }
        if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;
        double rhat_v;
        {
            double q[1] = {0.0}, o[1];
            for (int64_t rbase = warp * rows_per_warp; rbase < n; rbase += nwarps * rows_per_warp) {
                const int64_t row = rbase + lane / kKVec;
                const double sv = csr_row<kBicgVec, kBicgUnroll>(a, row, sub, ph);
                if (row < n && sub == 0) {
                    v[row] = sv;
                    q[0] += rh[row] * sv;
                }
            }
            if (!reduce<1>(a, turn, q, o)) return;
            rhat_v = o[0];
        }
        if (fabs(rhat_v) < 1e-40) {
            breakdown = 1;
            break;
        }
        alpha = rho / rhat_v;
        double s_norm;
        {
            double q[1] = {0.0}, o[1];
            for (int64_t i = tid; i < n; i += nth) {
                const double si = r[i] - alpha * v[i];
                s[i] = si;
                sh[i] = si * a.dinv[i];
                q[0] += si * si;
            }
            if (!reduce<1>(a, turn, q, o)) return;
            s_norm = sqrt(o[0]);
        }
        if (s_norm < a.tol * bnorm || s_norm < a.abs_tol) {
            for (int64_t i = tid; i < n; i += nth) a.x[i] += alpha * ph[i];
            final_res = s_norm;
            converged = 1;
            break;
        }
        double t_t, t_s;
        {
            double q[2] = {0.0, 0.0}, o[2];
            for (int64_t rbase = warp * rows_per_warp; rbase < n; rbase += nwarps * rows_per_warp) {
                const int64_t row = rbase + lane / kKVec;
                const double tv = csr_row<kBicgVec, kBicgUnroll>(a, row, sub, sh);
                if (row < n && sub == 0) {
                    t[row] = tv;
                    q[0] += tv * tv;
                    q[1] += tv * s[row];
                }
            }
            if (!reduce<2>(a, turn, q, o)) return;
            t_t = o[0];
            t_s = o[1];
        }
        if (fabs(t_t) < 1e-40) {
            breakdown = 1;
            break;
        }
        omega = t_s / t_t;
        {
            double q[1] = {0.0}, o[1];
            for (int64_t i = tid; i < n; i += nth) {
                a.x[i] += alpha * ph[i] + omega * sh[i];
                const double ri = s[i] - omega * t[i];
                r[i] = ri;
                q[0] += ri * ri;
            }
            if (!reduce<1>(a, turn, q, o)) return;
            final_res = sqrt(o[0]);
        }
        ++it;
        if (final_res < a.tol * bnorm || final_res < a.abs_tol) {
            converged = 1;
            break;
        }
        if (fabs(omega) < 1e-40) {
            breakdown = 1;
            break;
        }
    }
    if (tid == 0) *a.res = PcgResult{it, final_res, bnorm, converged, breakdown, 0};
}

// ------------------------------------------------------------------ GMRES(m) (iterative.rs:333-467)
__device__ __forceinline__ void givens(double a, double b, double& c, double& s, double& rho) {
    if (fabs(b) < 1e-40) {
        c = 1.0;
        s = 0.0;
        rho = a;
    } else if (fabs(b) > fabs(a)) {
        const double tau = a / b;
        s = 1.0 / sqrt(1.0 + tau * tau);
        c = s * tau;
        rho = b * sqrt(1.0 + tau * tau);
    } else {
        const double tau = b / a;
        c = 1.0 / sqrt(1.0 + tau * tau);
        s = c * tau;
        rho = a * sqrt(1.0 + tau * tau);
    }
}

__global__ void __launch_bounds__(kKBS, 4) k_gmres(KrylovArgs a) {
    constexpr int kKVec = kGmresVec;
    extern __shared__ double sm[];
    const int m = a.restart;
    double* H = sm;                    // (m + 1) x m, H[i * m + j]
    double* cs = H + (m + 1) * m;      // m
    double* sn = cs + m;               // m
    double* g = sn + m;                // m + 1
    double* y = g + m + 1;             // m
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31, sub = lane % kKVec;
    const int64_t warp = tid >> 5, nwarps = nth >> 5;
    constexpr int rows_per_warp = 32 / kKVec;
    const int64_t n = a.n;
    double *r = a.w[0], *w = a.w[1], *z = a.w[2];
    auto Vj = [&](int j) { return a.V + (size_t)j * n; };
    int turn = 0;
    init_dinv(a, tid, nth);
    double bnorm;
    {
        double q[1] = {0.0}, o[1];
        for (int64_t i = tid; i < n; i += nth) {
            a.x[i] = 0.0;
            q[0] += a.b[i] * a.b[i];
        }
        if (!reduce<1>(a, turn, q, o)) return;
        bnorm = sqrt(o[0]);
    }
    if (bnorm < 1e-25) {
        if (tid == 0) *a.res = PcgResult{0, 0.0, bnorm, 1, 0, 0};
        return;
    }
    long long total = 0;
    int converged = 0;
    double final_res = bnorm;
    while (total < a.max_it) {
        // r = b - A x and its norm (x complete: barrier at the end of the previous cycle)
        double r_norm;
        {
            double q[1] = {0.0}, o[1];
            for (int64_t rbase = warp * rows_per_warp; rbase < n; rbase += nwarps * rows_per_warp) {
                const int64_t row = rbase + lane / kKVec;
                const double ax = csr_row<kGmresVec, kGmresUnroll>(a, row, sub, a.x);
                if (row < n && sub == 0) {
                    const double ri = a.b[row] - ax;
                    r[row] = ri;
                    q[0] += ri * ri;
                }
            }
            if (!reduce<1>(a, turn, q, o)) return;
            r_norm = sqrt(o[0]);
        }
        final_res = r_norm;
        if (r_norm < a.tol * bnorm || r_norm < a.abs_tol) {
            converged = 1;
            break;
        }
        for (int64_t i = tid; i < n; i += nth) Vj(0)[i] = r[i] / r_norm;
        for (int q = threadIdx.x; q < (m + 1) * m; q += blockDim.x) H[q] = 0.0;
        for (int q = threadIdx.x; q < m; q += blockDim.x) cs[q] = sn[q] = y[q] = 0.0;
        for (int q = threadIdx.x; q <= m; q += blockDim.x) g[q] = 0.0;
        __syncthreads();
        if (threadIdx.x == 0) g[0] = r_norm;
        int k = 0;
        for (int j = 0; j < m; ++j) {
            if (total >= a.max_it) break;
            // z = M^-1 v_j (same thread wrote v_j[i]), then w = A z with h_0j = v_0 . w
            for (int64_t i = tid; i < n; i += nth) z[i] = Vj(j)[i] * a.dinv[i];
            if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;
            double hij;
            {
                double q[1] = {0.0}, o[1];
                const double* v0 = Vj(0);
                for (int64_t rbase = warp * rows_per_warp; rbase < n; rbase += nwarps * rows_per_warp) {
                    const int64_t row = rbase + lane / kKVec;
                    const double wv = csr_row<kGmresVec, kGmresUnroll>(a, row, sub, z);
                    if (row < n && sub == 0) {
                        w[row] = wv;
                        q[0] += v0[row] * wv;
                    }
                }
                if (!reduce<1>(a, turn, q, o)) return;
                hij = o[0];
            }
            // modified Gram-Schmidt: w -= h_ij v_i, fused with the next dot (or with ||w|| after the last)
            for (int i = 0; i <= j; ++i) {
                if (threadIdx.x == 0) H[i * m + j] = hij;
                const double* vi = Vj(i);
                const double* vn = i < j ? Vj(i + 1) : nullptr;
                double q[1] = {0.0}, o[1];
                for (int64_t l = tid; l < n; l += nth) {
                    const double wl = w[l] - hij * vi[l];
                    w[l] = wl;
                    q[0] += vn ? vn[l] * wl : wl * wl;
                }
                if (!reduce<1>(a, turn, q, o)) return;
                hij = i < j ? o[0] : sqrt(o[0]);
            }
            const double hnext = hij;  // h_{j+1,j} = ||w||
            double* vj1 = Vj(j + 1);
            if (fabs(hnext) > 1e-40)
                for (int64_t l = tid; l < n; l += nth) vj1[l] = w[l] / hnext;
            else
                for (int64_t l = tid; l < n; l += nth) vj1[l] = 0.0;
            __syncthreads();
            if (threadIdx.x == 0) {
                H[(j + 1) * m + j] = hnext;
                for (int i = 0; i < j; ++i) {
                    const double temp = cs[i] * H[i * m + j] + sn[i] * H[(i + 1) * m + j];
                    H[(i + 1) * m + j] = -sn[i] * H[i * m + j] + cs[i] * H[(i + 1) * m + j];
                    H[i * m + j] = temp;
                }
                double c, s, rho;
                givens(H[j * m + j], H[(j + 1) * m + j], c, s, rho);
                cs[j] = c;
                sn[j] = s;
                H[j * m + j] = rho;
                H[(j + 1) * m + j] = 0.0;
                const double temp = cs[j] * g[j];
                g[j + 1] = -sn[j] * g[j];
                g[j] = temp;
            }
            __syncthreads();
            k = j + 1;
            ++total;
            final_res = fabs(g[k]);
            if (final_res < a.tol * bnorm || final_res < a.abs_tol) break;
        }
        // y = H(1:k,1:k)^-1 g(1:k) by back-substitution, then x += M^-1 (V y)
        if (threadIdx.x == 0) {
            for (int i = k - 1; i >= 0; --i) {
                double sum = 0.0;
                for (int jj = i + 1; jj < k; ++jj) sum += H[i * m + jj] * y[jj];
                if (fabs(H[i * m + i]) < 1e-40) break;
                y[i] = (g[i] - sum) / H[i * m + i];
            }
        }
        __syncthreads();
        for (int64_t l = tid; l < n; l += nth) {
            double dy = 0.0;
            for (int jj = 0; jj < k; ++jj) dy += Vj(jj)[l] * y[jj];
            a.x[l] += dy * a.dinv[l];
        }
        if (!grid_barrier(a.gs, gridDim.x, a.timeout_ns)) return;
        if (final_res < a.tol * bnorm || final_res < a.abs_tol) {
            converged = 1;
            break;
        }
    }
    if (tid == 0) *a.res = PcgResult{total, final_res, bnorm, converged, 0, 0};
}

size_t gmres_smem(int m) { return sizeof(double) * ((size_t)(m + 1) * m + 4 * (size_t)m + 1); }

template <class Kernel>
int krylov_solve(geo_ctx* ctx, const geo_csr* A, const double* b, const geo_cg_opts* opts, int restart, double* x,
                 geo_solver_stats* stats, Kernel kernel, int nwork, bool gmres, const char* name) {
    GEO_CHECK_ARG(ctx && A && b && x, "NULL argument");
    GEO_CHECK_ARG(A->n_rows == A->n_cols, "matrix must be square");
    geo_cg_opts o;
    cg_opts_fill(opts, o);
    GEO_CHECK_ARG(o.max_iterations >= 0, "max_iterations must be >= 0");
    if (gmres) GEO_CHECK_ARG(restart >= 1 && restart <= kMaxRestart, "GMRES restart must be in 1..64");
    cudaStream_t s = ctx->stream;
    const int64_t n = A->n_rows;
    const int64_t np = (n + 31) / 32 * 32;
    DevBuf<double> tb, work((size_t)(2 + nwork) * np + (gmres ? (size_t)(restart + 1) * np : 0));
    const double* db = stage_in(b, n, tb, s);
    const size_t smem = gmres ? gmres_smem(restart) : 0;
    if (gmres) GEO_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int nb = persistent_blocks(ctx, kernel, kKBS, smem);
    PcgScratch sc;
    sc.ensure(nb);
    KrylovArgs args{};
    args.indptr = A->indptr.p;
    args.indices = A->indices.p;
    args.data = A->data.p;
    args.n = n;
    args.b = db;
    args.x = work.p;
    args.dinv = work.p + np;
    for (int k = 0; k < nwork; ++k) args.w[k] = work.p + (size_t)(2 + k) * np;
    args.V = gmres ? work.p + (size_t)(2 + nwork) * np : nullptr;
    args.part[0] = sc.slot(0, nb);
    args.part[1] = sc.slot(1, nb);
    args.gs = sc.gs.p;
    args.res = sc.res.p;
    args.timeout_ns = (unsigned long long)(o.timeout_seconds * 1e9);
    args.max_it = o.max_iterations;
    args.restart = restart;
    args.tol = o.tolerance;
    args.abs_tol = o.abs_tolerance;
    args.use_prec = o.use_preconditioner;
    GEO_CUDA(cudaMemsetAsync(sc.gs.p, 0, sizeof(GridSync), s));
    GEO_CUDA(cudaMemsetAsync(sc.res.p, 0, sizeof(PcgResult), s));
    GEO_CUDA(cudaEventRecord(ctx->ev0, s));
    launch_persistent(ctx, kernel, kKBS, smem, args, nb);
    GEO_CUDA(cudaEventRecord(ctx->ev1, s));
    PcgResult r{};
    GridSync gsync{};
    GEO_CUDA(cudaMemcpyAsync(&r, sc.res.p, sizeof(r), cudaMemcpyDeviceToHost, s));
    GEO_CUDA(cudaMemcpyAsync(&gsync, sc.gs.p, sizeof(gsync), cudaMemcpyDeviceToHost, s));
    copy_out(x, work.p, n, s);
    sync(ctx, name);
    float ms = 0.f;
    GEO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (gsync.error & DEV_ERR_TIMEOUT) {
        fill_stats(stats, r, ms * 1e-3, GEO_ERR_TIMEOUT);
        fail(GEO_ERR_TIMEOUT, std::string(name) + ": grid barrier timed out");
    }
    const int status = r.converged ? GEO_OK : (r.breakdown ? GEO_ERR_BREAKDOWN : GEO_NOT_CONVERGED);
    fill_stats(stats, r, ms * 1e-3, status);
    if (stats) stats->kernel_launches = 1;
    if (status != GEO_OK) {
        record_error(ctx, status, std::string(name) + (r.breakdown ? ": breakdown (a |denominator| < 1e-40)"
                                                                   : ": did not converge"));
        return status;
    }
    return GEO_OK;
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

int geo_bicgstab_solve(geo_ctx* ctx, const geo_csr* A, const double* b, const geo_cg_opts* opts, double* x,
                       geo_solver_stats* stats) {
    GEO_API_BEGIN(ctx)
    return krylov_solve(ctx, A, b, opts, 0, x, stats, k_bicgstab, 8, false, "geo_bicgstab_solve");
    GEO_API_END
}

int geo_gmres_solve(geo_ctx* ctx, const geo_csr* A, const double* b, const geo_cg_opts* opts, int32_t restart,
                    double* x, geo_solver_stats* stats) {
    GEO_API_BEGIN(ctx)
    return krylov_solve(ctx, A, b, opts, restart, x, stats, k_gmres, 3, true, "geo_gmres_solve");
    GEO_API_END
}

}  // extern "C"
