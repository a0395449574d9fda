// Host construction of the element-patch layout (see patches.h).
#include "patches.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include <omp.h>

namespace geo {

namespace {

inline uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

}  // namespace

void build_patches(int64_t N, const double* xyz, int64_t E, const int32_t* conn, PatchLayout& L) {
    L.n_elem = E;
    L.n_nodes = N;
    // ---- Morton order of element centroids (vertices 0..3)
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t n = 0; n < N; ++n)
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::min(lo[c], xyz[3 * n + c]);
            hi[c] = std::max(hi[c], xyz[3 * n + c]);
        }
    double sc[3];
    for (int c = 0; c < 3; ++c) sc[c] = hi[c] > lo[c] ? (double)((1 << 21) - 1) / (hi[c] - lo[c]) : 0.0;
    std::vector<std::pair<uint64_t, int32_t>> key(E);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; ++e) {
        double cen[3] = {0, 0, 0};
        for (int v = 0; v < 4; ++v)
            for (int c = 0; c < 3; ++c) cen[c] += 0.25 * xyz[3 * (int64_t)conn[10 * e + v] + c];
        uint64_t q[3];
        for (int c = 0; c < 3; ++c) q[c] = (uint64_t)std::llround((cen[c] - lo[c]) * sc[c]);
        key[e] = {spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2, (int32_t)e};
    }
    std::sort(key.begin(), key.end());
    L.eperm.resize(E);
    for (int64_t e = 0; e < E; ++e) L.eperm[e] = key[e].second;
    key.clear();
    key.shrink_to_fit();

    // ---- greedy patches + first-touch node numbering
    L.ninv.assign(N, -1);
    L.nperm.resize(N);
    std::vector<int32_t> stamp(N, -1);  // last patch that counted the node
    L.patch_elem.clear();
    L.patch_own.clear();
    L.patch_elem.push_back(0);
    L.patch_own.push_back(0);
    int32_t next_node = 0;
    int32_t patch = 0;
    int cur_elems = 0, cur_nodes = 0;
    for (int64_t ne = 0; ne < E; ++ne) {
        const int32_t* c = conn + 10 * (int64_t)L.eperm[ne];
        int fresh = 0;
        for (int l = 0; l < 10; ++l) {
            bool dup = false;
            for (int k = 0; k < l; ++k) dup |= c[k] == c[l];
            if (!dup && stamp[c[l]] != patch) ++fresh;
        }
        if (cur_elems > 0 && (cur_elems + 1 > kPatchElems || cur_nodes + fresh > kPatchNodes)) {
            L.patch_elem.push_back((int32_t)ne);
            L.patch_own.push_back(next_node);
            ++patch;
            cur_elems = 0;
            cur_nodes = 0;
            fresh = 0;
            for (int l = 0; l < 10; ++l) {
                bool dup = false;
                for (int k = 0; k < l; ++k) dup |= c[k] == c[l];
                if (!dup) ++fresh;
            }
        }
        for (int l = 0; l < 10; ++l) {
            const int32_t n = c[l];
            if (stamp[n] != patch) {
                stamp[n] = patch;
                ++cur_nodes;
            }
            if (L.ninv[n] < 0) {
                L.ninv[n] = next_node;
                L.nperm[next_node] = n;
                ++next_node;
            }
        }
        ++cur_elems;
    }
    L.patch_elem.push_back((int32_t)E);
    L.patch_own.push_back(next_node);
    L.n_patches = (int64_t)L.patch_elem.size() - 1;
    if (next_node != N) throw std::runtime_error("mesh has nodes that no element references");

    // ---- foreign lists, local connectivity, shared flags
    const int64_t P = L.n_patches;
    L.patch_foreign.assign(P + 1, 0);
    std::vector<std::vector<int32_t>> fl(P);
    L.lconn.resize((size_t)10 * E);
    L.shared.assign(N, 0);
    int max_local = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : max_local)
    for (int64_t p = 0; p < P; ++p) {
        const int32_t own0 = L.patch_own[p], own1 = L.patch_own[p + 1];
        std::vector<int32_t>& f = fl[p];
        for (int32_t ne = L.patch_elem[p]; ne < L.patch_elem[p + 1]; ++ne) {
            const int32_t* c = conn + 10 * (int64_t)L.eperm[ne];
            for (int l = 0; l < 10; ++l) {
                const int32_t nn = L.ninv[c[l]];
                if (nn < own0) f.push_back(nn);
            }
        }
        std::sort(f.begin(), f.end());
        f.erase(std::unique(f.begin(), f.end()), f.end());
        const int32_t n_own = own1 - own0;
        for (int32_t ne = L.patch_elem[p]; ne < L.patch_elem[p + 1]; ++ne) {
            const int32_t* c = conn + 10 * (int64_t)L.eperm[ne];
            for (int l = 0; l < 10; ++l) {
                const int32_t nn = L.ninv[c[l]];
                int32_t loc;
                if (nn >= own0) {
                    loc = nn - own0;
                } else {
                    loc = n_own + (int32_t)(std::lower_bound(f.begin(), f.end(), nn) - f.begin());
                }
                L.lconn[(size_t)l * E + ne] = (uint16_t)loc;
            }
        }
        max_local = std::max(max_local, n_own + (int)f.size());
    }
    L.max_local = max_local;
    if (max_local > kPatchNodes) throw std::runtime_error("patch exceeds its node budget");
    for (int64_t p = 0; p < P; ++p) {
        L.patch_foreign[p + 1] = L.patch_foreign[p] + (int32_t)fl[p].size();
        for (int32_t n : fl[p]) L.shared[n] = 1;
    }
    L.foreign.resize(L.patch_foreign[P]);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < P; ++p)
        std::copy(fl[p].begin(), fl[p].end(), L.foreign.begin() + L.patch_foreign[p]);
}

}  // namespace geo
