// GPU construction of the element-patch layout (see patches.h). All steps are
// data-parallel: Morton keys + radix sort for the element order, atomicMin of
// the first-touch position for the node order, a sort of each patch's own
// candidates in shared memory (one block per patch) for the per-patch foreign
// lists, binary searches for the local indices.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>

#include "patches.h"

namespace geo {
namespace {

inline unsigned nb(int64_t n, int bs = 256) { return (unsigned)std::max<int64_t>(1, cdiv(n, bs)); }

__device__ __forceinline__ uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(const double* __restrict__ xyz, const int32_t* __restrict__ conn, int64_t N, int64_t E,
                         const double* __restrict__ lohi, uint64_t* __restrict__ key, int32_t* __restrict__ idx) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    uint64_t q[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double cen = 0.0;
#pragma unroll
        for (int v = 0; v < 4; ++v) cen += 0.25 * xyz[c * N + conn[v * E + e]];
        const double lo = lohi[c], hi = lohi[3 + c];
        const double sc = hi > lo ? (double)((1 << 21) - 1) / (hi - lo) : 0.0;
        q[c] = (uint64_t)llrint(fmin(fmax((cen - lo) * sc, 0.0), (double)((1 << 21) - 1)));
    }
    key[e] = spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2;
    idx[e] = (int32_t)e;
}

__global__ void k_bbox(const double* __restrict__ xyz, int64_t N, unsigned long long* __restrict__ out) {
    // out[0..2] = ordered-int of min, out[3..5] = ordered-int of max
    double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = xyz[c * N + i];
            lo[c] = fmin(lo[c], v);
            hi[c] = fmax(hi[c], v);
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fmin(lo[c], __shfl_down_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_down_sync(0xffffffffu, hi[c], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        // map doubles to order-preserving unsigned keys
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            unsigned long long a = (unsigned long long)__double_as_longlong(lo[c]);
            a = (a >> 63) ? ~a : (a | 0x8000000000000000ull);
            atomicMin(&out[c], a);
            unsigned long long b = (unsigned long long)__double_as_longlong(hi[c]);
            b = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
            atomicMax(&out[3 + c], b);
        }
    }
}

__global__ void k_bbox_decode(const unsigned long long* in, double* lohi) {
    const int c = threadIdx.x;
    if (c >= 6) return;
    unsigned long long a = in[c];
    a = (a >> 63) ? (a & 0x7fffffffffffffffull) : ~a;
    lohi[c] = __longlong_as_double((long long)a);
}

__global__ void k_first_touch(const int32_t* __restrict__ conn, const int32_t* __restrict__ eperm, int64_t E,
                              int32_t* __restrict__ ft) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= E * 10) return;
    const int64_t ne = t / 10;
    const int l = (int)(t % 10);
    atomicMin(&ft[conn[l * E + eperm[ne]]], (int32_t)t);
}

__global__ void k_fill_max(int32_t* v, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = INT_MAX;
}

__global__ void k_iota(int32_t* v, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

__global__ void k_inverse(const int32_t* __restrict__ perm, int64_t n, int32_t* __restrict__ inv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) inv[perm[i]] = (int32_t)i;
}

// patch_elem[p] = min(p*PE, E); patch_own[p] = #new nodes with first touch < p*PE*10
__global__ void k_patch_bounds(const int32_t* __restrict__ ft_sorted, int64_t N, int64_t E, int P,
                               int32_t* __restrict__ pe, int32_t* __restrict__ po) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > P) return;
    const int64_t e0 = std::min<int64_t>((int64_t)p * kPatchElems, E);
    pe[p] = (int32_t)e0;
    const int64_t key = e0 * 10;
    int64_t lo = 0, hi = N;
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if ((int64_t)ft_sorted[m] < key) lo = m + 1;
        else hi = m;
    }
    po[p] = (int32_t)lo;
}

// key = patch << 32 | new node for every foreign incidence, ~0 otherwise
// Foreign nodes of a patch: the distinct node ids below the patch's own range that
// its elements reference, in ascending order. One block per patch gathers the
// candidates of its (at most 10 * kPatchElems) incidences into shared memory,
// sorts them there (bitonic network) and marks the first of every run of equal ids.
constexpr int kForeignBS = 256;
constexpr int kForeignCap = 4096;  // power of two >= 10 * kPatchElems
static_assert(kForeignCap >= 10 * kPatchElems, "foreign candidate buffer too small");

__device__ int patch_foreign_sorted(const int32_t* __restrict__ conn, const int32_t* __restrict__ eperm,
                                    const int32_t* __restrict__ ninv, const int32_t* __restrict__ po, int64_t E,
                                    int* s_keys) {
    __shared__ int s_n;
    const int p = blockIdx.x;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const int32_t own0 = po[p];
    const int64_t e0 = (int64_t)p * kPatchElems, e1 = min(E, e0 + kPatchElems);
    const int n_inc = (int)((e1 - e0) * 10);
    for (int t = threadIdx.x; t < n_inc; t += blockDim.x) {
        const int64_t ne = e0 + t / 10;
        const int l = t % 10;
        const int32_t nn = ninv[conn[(int64_t)l * E + eperm[ne]]];
        if (nn < own0) s_keys[atomicAdd(&s_n, 1)] = nn;
    }
    __syncthreads();
    const int n = s_n;
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = n + threadIdx.x; i < m; i += blockDim.x) s_keys[i] = INT32_MAX;
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int a = s_keys[i], b = s_keys[ixj];
                    if (((i & k) == 0) ? (a > b) : (a < b)) {
                        s_keys[i] = b;
                        s_keys[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    return n;
}

// Block-wide exclusive scan of one int per thread (blockDim.x == kForeignBS); total in *total.
__device__ int block_exclusive_scan(int v, int* total) {
    __shared__ int s_warp[kForeignBS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    int base = 0, sum = 0;
    for (int w = 0; w < kForeignBS / 32; ++w) {
        if (w < warp) base += s_warp[w];
        sum += s_warp[w];
    }
    __syncthreads();
    *total = sum;
    return base + x - v;
}

// Pass 1 (write == false): cnt[p] = number of distinct foreign nodes of patch p.
// Pass 2 (write == true): foreign[pf[p] ..] = those nodes in ascending order, shared[node] = 1.
template <bool WRITE>
__global__ void __launch_bounds__(kForeignBS) k_patch_foreign_lists(
    const int32_t* __restrict__ conn, const int32_t* __restrict__ eperm, const int32_t* __restrict__ ninv,
    const int32_t* __restrict__ po, int64_t E, int32_t* __restrict__ cnt, const int32_t* __restrict__ pf,
    int32_t* __restrict__ foreign, uint8_t* __restrict__ shared) {
    __shared__ int s_keys[kForeignCap];
    const int n = patch_foreign_sorted(conn, eperm, ninv, po, E, s_keys);
    // each thread takes a contiguous chunk of the sorted candidates
    constexpr int kPer = kForeignCap / kForeignBS;
    const int i0 = threadIdx.x * kPer;
    int c = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const int i = i0 + q;
        if (i < n && (i == 0 || s_keys[i] != s_keys[i - 1])) ++c;
    }
    int total = 0;
    int at = block_exclusive_scan(c, &total);
    if (!WRITE) {
        if (threadIdx.x == 0) cnt[blockIdx.x] = total;
        return;
    }
    const int32_t base = pf[blockIdx.x];
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const int i = i0 + q;
        if (i < n && (i == 0 || s_keys[i] != s_keys[i - 1])) {
            const int nn = s_keys[i];
            foreign[base + at++] = nn;
            shared[nn] = 1;
        }
    }
}

__global__ void k_local_conn(const int32_t* __restrict__ conn, const int32_t* __restrict__ eperm,
                             const int32_t* __restrict__ ninv, const int32_t* __restrict__ po,
                             const int32_t* __restrict__ pf, const int32_t* __restrict__ foreign, int64_t E,
                             uint16_t* __restrict__ lconn, int* __restrict__ err) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= E * 10) return;
    const int64_t ne = t / 10;
    const int l = (int)(t % 10);
    const int32_t nn = ninv[conn[l * E + eperm[ne]]];
    const int p = (int)(ne / kPatchElems);
    const int32_t own0 = po[p], nown = po[p + 1] - own0;
    int64_t loc;
    if (nn >= own0) {
        loc = nn - own0;
        if (loc >= nown) atomicOr(err, DEV_ERR_BOUNDS);
    } else {
        int64_t lo = pf[p], hi = pf[p + 1];
        while (lo < hi) {
            const int64_t m = (lo + hi) >> 1;
            if (foreign[m] < nn) lo = m + 1;
            else hi = m;
        }
        if (lo >= pf[p + 1] || foreign[lo] != nn) atomicOr(err, DEV_ERR_BOUNDS);
        loc = nown + (lo - pf[p]);
    }
    const int64_t slot = loc + (loc >> 5);  // patch_slot
    if (slot > 65535) atomicOr(err, DEV_ERR_BOUNDS);
    lconn[(int64_t)l * E + ne] = (uint16_t)slot;
}

__global__ void k_local_sizes(const int32_t* po, const int32_t* pf, int P, int* out) {
    int m = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
        m = max(m, (po[p + 1] - po[p]) + (pf[p + 1] - pf[p]));
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Orders each patch's elements so that every aligned group of 32 has pairwise
// node-disjoint elements where possible (greedy in element order), making the
// shared-memory accumulation of a warp conflict-free. One warp per patch. The
// lanes test 32 consecutive candidates at once against the nodes the group
// already uses; the lowest passing lane's element is the one a sequential scan
// would take next, so it is taken, its nodes marked, and the lanes above it test
// again. The result equals the sequential greedy's element for element.
constexpr int kOrderWarps = 4;
__global__ void __launch_bounds__(32 * kOrderWarps)
k_patch_order(const uint16_t* __restrict__ lconn, int64_t E, const int32_t* __restrict__ pe, int P,
              int32_t* __restrict__ wperm) {
    __shared__ uint16_t sl[kOrderWarps][10][kPatchElems];
    __shared__ uint32_t used[kOrderWarps][(patch_slot(10 * kPatchElems) + 31) / 32];
    __shared__ uint8_t taken[kOrderWarps][kPatchElems];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * kOrderWarps + w;
    if (p >= P) return;  // warp-uniform
    const int e0 = pe[p], n_el = pe[p + 1] - e0;
    int nloc = 0;
    for (int t = lane; t < 10 * n_el; t += 32) {
        const uint16_t v = lconn[(int64_t)(t / n_el) * E + e0 + t % n_el];
        sl[w][t / n_el][t % n_el] = v;
        nloc = max(nloc, (int)v + 1);
    }
    nloc = __reduce_max_sync(0xffffffffu, nloc);
    for (int j = lane; j < n_el; j += 32) taken[w][j] = 0;
    const int words = (nloc + 31) / 32;
    uint32_t* uw = used[w];
    // element j (< n_el) shares no node with the group so far
    auto disjoint = [&](int j) {
        for (int l = 0; l < 10; ++l) {
            const int u = sl[w][l][j];
            if ((uw[u >> 5] >> (u & 31)) & 1u) return false;
        }
        return true;
    };
    int out = 0;  // warp-uniform
    while (out < n_el) {
        for (int k = lane; k < words; k += 32) uw[k] = 0u;
        __syncwarp();
        int cnt = 0;
        for (int j0 = 0; j0 < n_el && cnt < 32; j0 += 32) {
            const int j = j0 + lane;
            bool cand = j < n_el && !taken[w][j] && disjoint(j);
            unsigned m = __ballot_sync(0xffffffffu, cand);
            while (m != 0u && cnt < 32) {
                const int L = __ffs(m) - 1;
                if (lane == L) {  // the only writer of the group's node bits
                    for (int l = 0; l < 10; ++l) {
                        const int u = sl[w][l][j];
                        uw[u >> 5] |= 1u << (u & 31);
                    }
                    taken[w][j] = 1;
                    wperm[e0 + out] = e0 + j;
                }
                ++out;
                ++cnt;
                __syncwarp();
                cand = cand && lane > L && disjoint(j);
                m = __ballot_sync(0xffffffffu, cand);
            }
        }
        // keep groups aligned with warps: top up with the next untaken elements
        for (int j0 = 0; j0 < n_el && cnt < 32 && out < n_el; j0 += 32) {
            const int j = j0 + lane;
            unsigned m = __ballot_sync(0xffffffffu, j < n_el && !taken[w][j]);
            while (m != 0u && cnt < 32 && out < n_el) {
                const int L = __ffs(m) - 1;
                if (lane == L) {
                    taken[w][j] = 1;
                    wperm[e0 + out] = e0 + j;
                }
                ++out;
                ++cnt;
                m &= m - 1u;
            }
            __syncwarp();
        }
    }
}

// Applies the within-patch order: eperm2[ne] = eperm[wperm[ne]] and the
// patch-major paired connectivity (see PatchLayout::lc).
__global__ void k_apply_order(const int32_t* __restrict__ wperm, const int32_t* __restrict__ eperm,
                              const uint16_t* __restrict__ lconn, int64_t E, int P, int32_t* __restrict__ eperm2,
                              uint32_t* __restrict__ lc) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)P * kPatchElems) return;
    const int64_t p = t / kPatchElems, j = t % kPatchElems;
    const int64_t ne = t;
    if (ne < E) {
        const int64_t src = wperm[ne];
        eperm2[ne] = eperm[src];
        for (int l2 = 0; l2 < 5; ++l2)
            lc[(p * 5 + l2) * kPatchElems + j] =
                (uint32_t)lconn[(int64_t)(2 * l2) * E + src] | (uint32_t)lconn[(int64_t)(2 * l2 + 1) * E + src] << 16;
    } else {
        for (int l2 = 0; l2 < 5; ++l2) lc[(p * 5 + l2) * kPatchElems + j] = 0u;
    }
}

template <class F>
void cub_call(cudaStream_t s, F&& f) {
    size_t bytes = 0;
    GEO_CUDA(f((void*)nullptr, bytes));
    DevBuf<unsigned char> tmp(bytes + 16);
    GEO_CUDA(f((void*)tmp.p, bytes));
    GEO_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

void build_patches(cudaStream_t s, int64_t N, const double* xyz, int64_t E, const int32_t* conn, PatchLayout& L) {
    L.n_elem = E;
    L.n_nodes = N;
    const int P = (int)cdiv(E, kPatchElems);
    L.n_patches = P;
    // ---- element order: Morton code of the vertex centroid
    DevBuf<unsigned long long> bb(6);
    DevBuf<double> lohi(6);
    {
        const unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
        GEO_CUDA(cudaMemcpyAsync(bb.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
        k_bbox<<<std::min<unsigned>(nb(N), 2048), 256, 0, s>>>(xyz, N, bb.p);
        k_bbox_decode<<<1, 32, 0, s>>>(bb.p, lohi.p);
    }
    {
        DevBuf<uint64_t> k0(E), k1(E);
        DevBuf<int32_t> i0(E);
        L.eperm.alloc(E);
        k_morton<<<nb(E), 256, 0, s>>>(xyz, conn, N, E, lohi.p, k0.p, i0.p);
        cub_call(s, [&](void* t, size_t& b) {
            return cub::DeviceRadixSort::SortPairs(t, b, k0.p, k1.p, i0.p, L.eperm.p, E, 0, 63, s);
        });
    }
    // ---- node order: first touch over (patch-ordered element, local node)
    L.nperm.alloc(N);
    L.ninv.alloc(N);
    DevBuf<int32_t> ft(N), ft_sorted(N);
    {
        DevBuf<int32_t> ids(N);
        k_fill_max<<<nb(N), 256, 0, s>>>(ft.p, N);
        k_first_touch<<<nb(E * 10), 256, 0, s>>>(conn, L.eperm.p, E, ft.p);
        k_iota<<<nb(N), 256, 0, s>>>(ids.p, N);
        cub_call(s, [&](void* t, size_t& b) {
            return cub::DeviceRadixSort::SortPairs(t, b, ft.p, ft_sorted.p, ids.p, L.nperm.p, N, 0, 32, s);
        });
        int32_t last = 0;
        GEO_CUDA(cudaMemcpy(&last, ft_sorted.p + N - 1, sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (last >= (int32_t)(E * 10)) fail(GEO_ERR_UNSUPPORTED, "mesh has nodes that no element references");
        k_inverse<<<nb(N), 256, 0, s>>>(L.nperm.p, N, L.ninv.p);
    }
    L.patch_elem.alloc(P + 1);
    L.patch_own.alloc(P + 1);
    k_patch_bounds<<<nb(P + 1), 256, 0, s>>>(ft_sorted.p, N, E, P, L.patch_elem.p, L.patch_own.p);
    // ---- foreign lists
    L.patch_foreign.alloc(P + 1);
    L.shared.alloc(N);
    GEO_CUDA(cudaMemsetAsync(L.shared.p, 0, N, s));
    int64_t nf = 0;
    {
        // per patch in shared memory: count, offsets by scan, then the sorted lists
        DevBuf<int32_t> cnt(P + 1);
        GEO_CUDA(cudaMemsetAsync(cnt.p + P, 0, sizeof(int32_t), s));
        k_patch_foreign_lists<false><<<(unsigned)P, kForeignBS, 0, s>>>(conn, L.eperm.p, L.ninv.p, L.patch_own.p, E,
                                                                       cnt.p, nullptr, nullptr, nullptr);
        cub_call(s, [&](void* t, size_t& b) {
            return cub::DeviceScan::ExclusiveSum(t, b, cnt.p, L.patch_foreign.p, P + 1, s);
        });
        int32_t total = 0;
        GEO_CUDA(cudaMemcpy(&total, L.patch_foreign.p + P, sizeof(int32_t), cudaMemcpyDeviceToHost));
        nf = total;
        L.foreign.alloc(std::max<int64_t>(nf, 1));
        k_patch_foreign_lists<true><<<(unsigned)P, kForeignBS, 0, s>>>(conn, L.eperm.p, L.ninv.p, L.patch_own.p, E,
                                                                      nullptr, L.patch_foreign.p, L.foreign.p,
                                                                      L.shared.p);
        GEO_CUDA(cudaGetLastError());
        GEO_CUDA(cudaStreamSynchronize(s));
    }
    // ---- local connectivity and patch-table size
    DevBuf<int> err(2);
    GEO_CUDA(cudaMemsetAsync(err.p, 0, 2 * sizeof(int), s));
    DevBuf<uint16_t> lconn(E * 10);
    k_local_conn<<<nb(E * 10), 256, 0, s>>>(conn, L.eperm.p, L.ninv.p, L.patch_own.p, L.patch_foreign.p,
                                           L.foreign.p, E, lconn.p, err.p);
    k_local_sizes<<<std::min<unsigned>(nb(P), 1024), 256, 0, s>>>(L.patch_own.p, L.patch_foreign.p, P, err.p + 1);
    GEO_CUDA(cudaGetLastError());
    int h[2] = {0, 0};
    GEO_CUDA(cudaMemcpyAsync(h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    GEO_CUDA(cudaStreamSynchronize(s));
    if (h[0]) fail(GEO_ERR_UNSUPPORTED, "patch-local index out of range while building the element patches");
    L.max_local = h[1] > 0 ? patch_slot(h[1] - 1) + 1 : 0;  // table size in slots
    // ---- conflict-avoiding element order inside each patch, patch-major connectivity
    {
        DevBuf<int32_t> wperm(E), eperm2(E);
        k_patch_order<<<(unsigned)cdiv(P, kOrderWarps), 32 * kOrderWarps, 0, s>>>(lconn.p, E, L.patch_elem.p, P,
                                                                                  wperm.p);
        L.lc.alloc((size_t)P * 5 * kPatchElems);
        k_apply_order<<<nb((int64_t)P * kPatchElems), 256, 0, s>>>(wperm.p, L.eperm.p, lconn.p, E, P, eperm2.p,
                                                                    L.lc.p);
        GEO_CUDA(cudaGetLastError());
        GEO_CUDA(cudaStreamSynchronize(s));
        L.eperm = std::move(eperm2);
    }
}

}  // namespace geo
