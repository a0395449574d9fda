// ImprovedMeshGenerator::generate_cube (mesh_generator_improved.rs:19-169), host code.
//
// Same node numbering and connectivity as the reference, bit for bit: vertices
// first (x fastest, then y, then z), then edge midpoints in first-touch order of
// the per-tet edge sequence e01 e12 e20 e03 e13 e23. The reference keys a HashMap
// by the sorted vertex pair; on the structured lattice every edge of the 6-tet
// (Kuhn) subdivision runs from a lattice corner in one of 7 non-negative
// directions, so a flat [7][n_vertices] table replaces the hash map.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "geo_fem.h"

namespace {

thread_local std::string t_err;

inline int64_t cube_nodes(int64_t nx, int64_t ny, int64_t nz) {
    const int64_t v = (nx + 1) * (ny + 1) * (nz + 1);
    const int64_t ex = nx * (ny + 1) * (nz + 1), ey = (nx + 1) * ny * (nz + 1),
                  ez = (nx + 1) * (ny + 1) * nz;
    const int64_t fxy = nx * ny * (nz + 1), fxz = nx * (ny + 1) * nz, fyz = (nx + 1) * ny * nz;
    return v + ex + ey + ez + fxy + fxz + fyz + nx * ny * nz;
}

}  // namespace

extern "C" {

int geo_generate_cube_size(int64_t nx, int64_t ny, int64_t nz, int64_t* n_nodes, int64_t* n_elem) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !n_nodes || !n_elem) return GEO_ERR_INVALID_ARG;
    *n_nodes = cube_nodes(nx, ny, nz);
    *n_elem = 6 * nx * ny * nz;
    return GEO_OK;
}

int geo_generate_cube(int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz,
                      double* xyz, int32_t* conn) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !xyz || !conn) return GEO_ERR_INVALID_ARG;
    const int64_t N = cube_nodes(nx, ny, nz);
    if (N >= (int64_t(1) << 31) || 60 * nx * ny * nz >= (int64_t(1) << 31)) return GEO_ERR_INVALID_ARG;
    const double dx = lx / (double)nx, dy = ly / (double)ny, dz = lz / (double)nz;
    const int64_t sx = 1, sy = nx + 1, sz = (nx + 1) * (ny + 1);
    const int64_t NV = sz * (nz + 1);
    int64_t next = 0;
    for (int64_t iz = 0; iz <= nz; ++iz)
        for (int64_t iy = 0; iy <= ny; ++iy)
            for (int64_t ix = 0; ix <= nx; ++ix) {
                xyz[3 * next] = (double)ix * dx;
                xyz[3 * next + 1] = (double)iy * dy;
                xyz[3 * next + 2] = (double)iz * dz;
                ++next;
            }
    // direction code of (v_hi - v_lo) in lattice strides
    auto dir_of = [&](int64_t d) -> int {
        if (d == sx) return 0;
        if (d == sy) return 1;
        if (d == sz) return 2;
        if (d == sx + sy) return 3;
        if (d == sx + sz) return 4;
        if (d == sy + sz) return 5;
        if (d == sx + sy + sz) return 6;
        return -1;
    };
    std::vector<int32_t> table((size_t)7 * NV, -1);
    auto midpoint = [&](int64_t a, int64_t b) -> int32_t {
        const int64_t lo = a < b ? a : b, hi = a < b ? b : a;
        const int d = dir_of(hi - lo);
        int32_t& slot = table[(size_t)d * NV + lo];
        if (slot < 0) {
            const double* pa = xyz + 3 * a;
            const double* pb = xyz + 3 * b;
            xyz[3 * next] = (pa[0] + pb[0]) / 2.0;
            xyz[3 * next + 1] = (pa[1] + pb[1]) / 2.0;
            xyz[3 * next + 2] = (pa[2] + pb[2]) / 2.0;
            slot = (int32_t)next++;
        }
        return slot;
    };
    int64_t e = 0;
    for (int64_t iz = 0; iz < nz; ++iz)
        for (int64_t iy = 0; iy < ny; ++iy)
            for (int64_t ix = 0; ix < nx; ++ix) {
                const int64_t v000 = ix * sx + iy * sy + iz * sz;
                const int64_t v100 = v000 + sx, v010 = v000 + sy, v110 = v000 + sx + sy;
                const int64_t v001 = v000 + sz, v101 = v001 + sx, v011 = v001 + sy, v111 = v001 + sx + sy;
                const int64_t tets[6][4] = {{v000, v100, v110, v111}, {v000, v100, v111, v101},
                                            {v000, v010, v110, v111}, {v000, v010, v111, v011},
                                            {v000, v001, v111, v101}, {v000, v001, v111, v011}};
                for (int t = 0; t < 6; ++t) {
                    const int64_t v0 = tets[t][0], v1 = tets[t][1];
                    int64_t v2 = tets[t][2], v3 = tets[t][3];
                    const double* p0 = xyz + 3 * v0;
                    const double* p1 = xyz + 3 * v1;
                    const double* p2 = xyz + 3 * v2;
                    const double* p3 = xyz + 3 * v3;
                    const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
                    const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
                    const double e3[3] = {p3[0] - p0[0], p3[1] - p0[1], p3[2] - p0[2]};
                    const double det = e1[0] * (e2[1] * e3[2] - e2[2] * e3[1]) +
                                       e1[1] * (e2[2] * e3[0] - e2[0] * e3[2]) +
                                       e1[2] * (e2[0] * e3[1] - e2[1] * e3[0]);
                    if (det < 0.0) {
                        const int64_t t2 = v2;
                        v2 = v3;
                        v3 = t2;
                    }
                    int32_t* c = conn + 10 * e;
                    c[0] = (int32_t)v0;
                    c[1] = (int32_t)v1;
                    c[2] = (int32_t)v2;
                    c[3] = (int32_t)v3;
                    c[4] = midpoint(v0, v1);
                    c[5] = midpoint(v1, v2);
                    c[6] = midpoint(v2, v0);
                    c[7] = midpoint(v0, v3);
                    c[8] = midpoint(v1, v3);
                    c[9] = midpoint(v2, v3);
                    ++e;
                }
            }
    if (next != N) {
        t_err = "internal node count mismatch";
        return GEO_ERR_INVALID_ARG;
    }
    return GEO_OK;
}

}  // extern "C"
