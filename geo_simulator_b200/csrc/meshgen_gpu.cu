// Structured Tet10 cube mesh built on the device: the drop-in for
// ImprovedMeshGenerator::generate_cube (mesh_generator_improved.rs:19-169) that
// leaves the mesh resident in the SoA layout the kernels read, with the node
// numbering, coordinates and connectivity of the host generator bit for bit.
//
// The reference numbers edge midpoints in the order its loop first touches them:
// hexes z-outer / x-inner, 6 tets per hex, edges e01 e12 e20 e03 e13 e23 of each
// tet (after the v2<->v3 orientation swap). On the lattice that order has a
// closed form, so no hash map and no atomics are needed:
//  * every tet of the 6-tet subdivision is a chain of hex corners, so each of
//    its edges runs from a corner l to a corner u whose bit set contains l's
//    (corner bit 0 = +x, 1 = +y, 2 = +z); the direction is m = l ^ u;
//  * the first hex to touch an edge is the lowest-numbered hex containing it:
//    the edge is "owned" by this hex iff, along every axis a not in m, the edge
//    lies on the hex's high face (bit a of l set) or the hex index along a is 0;
//  * so the number of midpoints a hex creates depends only on which of its
//    indices are 0, and the id of its first new midpoint is a closed-form prefix
//    sum over the hexes before it;
//  * within the hex, owned edges get consecutive ids at their first occurrence
//    in the tet/edge sequence.
// Kernel 1 (one thread per hex) writes the owned midpoints' coordinates and
// their ids into a [7][n_vertices] edge table; kernel 2 (one thread per tet)
// writes the 10 connectivity rows, coalesced, reading midpoint ids from the
// table. Coordinates use the host generator's arithmetic with explicitly
// rounded operations (no FMA contraction): vertex = (double)i * (l / n),
// midpoint = (a + b) / 2, and the orientation determinant's sign.
#include <algorithm>

#include "objects.h"

namespace geo {
namespace {

// Tets of one hex as corner codes, in the reference's order (mesh_generator_improved.rs:81-123):
// {0,1,3,7} {0,1,7,5} {0,2,3,7} {0,2,7,6} {0,4,7,5} {0,4,7,6}. Corner 0 opens every tet;
// corners 1..3 are packed 3 bits each, 9 bits per tet, so that lanes working on
// different tets read an immediate instead of divergent constant memory.
constexpr uint64_t pack_tet(int t, int a, int b, int c) {
    return (uint64_t)(a | (b << 3) | (c << 6)) << (9 * t);
}
constexpr uint64_t kHexTets = pack_tet(0, 1, 3, 7) | pack_tet(1, 1, 7, 5) | pack_tet(2, 2, 3, 7) |
                              pack_tet(3, 2, 7, 6) | pack_tet(4, 4, 7, 5) | pack_tet(5, 4, 7, 6);
__device__ __forceinline__ int tet_corner(int t, int k) {
    return k == 0 ? 0 : (int)((kHexTets >> (9 * t + 3 * (k - 1))) & 7u);
}
// Tet10 edge midpoints 4..9 as local vertex pairs (create_tet10, :126-169):
// (0,1) (1,2) (2,0) (0,3) (1,3) (2,3), 2 bits per vertex, 4 bits per edge
constexpr uint32_t kTetEdges = 0x0u | (0x1u << 2) | (0x1u << 4) | (0x2u << 6) | (0x2u << 8) | (0x0u << 10) |
                               (0x0u << 12) | (0x3u << 14) | (0x1u << 16) | (0x3u << 18) | (0x2u << 20) |
                               (0x3u << 22);
__device__ __forceinline__ int tet_edge(int k, int j) { return (int)((kTetEdges >> (4 * k + 2 * j)) & 3u); }
// direction code of an edge from its corner bit difference m (x=1, y=2, z=4), 4 bits
// per m: the host generator's order sx, sy, sz, sx+sy, sx+sz, sy+sz, sx+sy+sz
constexpr uint32_t kDirOfBits = (0u << 4) | (1u << 8) | (3u << 12) | (2u << 16) | (4u << 20) | (5u << 24) |
                                (6u << 28);
__device__ __forceinline__ int dir_of_bits(int m) { return (int)((kDirOfBits >> (4 * m)) & 15u); }

struct CubeGrid {
    int64_t nx, ny, nz;
    int64_t sy, sz;  // vertex strides (sx = 1)
    int64_t nv;      // vertices
    int64_t n_nodes, n_hex, n_elem;
    double dx, dy, dz;
};

// Midpoints created by a hex whose x/y/z index is 0 (bx/by/bz = 1) or not:
// body diagonal, three face diagonals (+1 each on a low boundary face) and the
// axis edges (x-edges (1+by)(1+bz), and so on).
__host__ __device__ __forceinline__ int64_t owned_count(int bx, int by, int bz) {
    return 1 + (1 + bz) + (1 + by) + (1 + bx) + (1 + by) * (1 + bz) + (1 + bx) * (1 + bz) + (1 + bx) * (1 + by);
}

__host__ __device__ __forceinline__ int64_t row_count(int64_t nx, int by, int bz) {
    return owned_count(1, by, bz) + (nx - 1) * owned_count(0, by, bz);
}

__host__ __device__ __forceinline__ int64_t plane_count(int64_t nx, int64_t ny, int bz) {
    return row_count(nx, 1, bz) + (ny - 1) * row_count(nx, 0, bz);
}

// Number of midpoints created by all hexes before hex (ix, iy, iz) in z-outer order.
__host__ __device__ __forceinline__ int64_t midpoints_before(int64_t ix, int64_t iy, int64_t iz, int64_t nx,
                                                             int64_t ny) {
    int64_t s = 0;
    if (iz > 0) s += plane_count(nx, ny, 1) + (iz - 1) * plane_count(nx, ny, 0);
    const int bz = iz == 0;
    if (iy > 0) s += row_count(nx, 1, bz) + (iy - 1) * row_count(nx, 0, bz);
    const int by = iy == 0;
    if (ix > 0) s += owned_count(1, by, bz) + (ix - 1) * owned_count(0, by, bz);
    return s;
}

__device__ __forceinline__ double coord(int64_t i, double d) { return __dmul_rn((double)i, d); }

struct HexCorners {
    double x0, x1, y0, y1, z0, z1;  // coordinates of the low / high lattice planes
    int64_t v000;
    __device__ __forceinline__ double x(int c) const { return (c & 1) ? x1 : x0; }
    __device__ __forceinline__ double y(int c) const { return (c & 2) ? y1 : y0; }
    __device__ __forceinline__ double z(int c) const { return (c & 4) ? z1 : z0; }
};

__device__ __forceinline__ HexCorners hex_corners(const CubeGrid& g, int64_t ix, int64_t iy, int64_t iz) {
    HexCorners h;
    h.x0 = coord(ix, g.dx);
    h.x1 = coord(ix + 1, g.dx);
    h.y0 = coord(iy, g.dy);
    h.y1 = coord(iy + 1, g.dy);
    h.z0 = coord(iz, g.dz);
    h.z1 = coord(iz + 1, g.dz);
    h.v000 = ix + iy * g.sy + iz * g.sz;
    return h;
}

__device__ __forceinline__ int64_t corner_id(const CubeGrid& g, const HexCorners& h, int c) {
    return h.v000 + (c & 1) + ((c >> 1) & 1) * g.sy + ((c >> 2) & 1) * g.sz;
}

// Tet corners in the reference's order, with v2/v3 swapped when the signed
// volume is negative (the determinant expanded along the first row, as the
// host generator computes it).
__device__ __forceinline__ void oriented_tet(const HexCorners& h, int t, int (&c)[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = tet_corner(t, k);
    double p[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        p[k][0] = h.x(c[k]);
        p[k][1] = h.y(c[k]);
        p[k][2] = h.z(c[k]);
    }
    double e1[3], e2[3], e3[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e1[a] = __dsub_rn(p[1][a], p[0][a]);
        e2[a] = __dsub_rn(p[2][a], p[0][a]);
        e3[a] = __dsub_rn(p[3][a], p[0][a]);
    }
    const double c0 = __dsub_rn(__dmul_rn(e2[1], e3[2]), __dmul_rn(e2[2], e3[1]));
    const double c1 = __dsub_rn(__dmul_rn(e2[2], e3[0]), __dmul_rn(e2[0], e3[2]));
    const double c2 = __dsub_rn(__dmul_rn(e2[0], e3[1]), __dmul_rn(e2[1], e3[0]));
    const double det = __dadd_rn(__dadd_rn(__dmul_rn(e1[0], c0), __dmul_rn(e1[1], c1)), __dmul_rn(e1[2], c2));
    if (det < 0.0) {
        const int t2 = c[2];
        c[2] = c[3];
        c[3] = t2;
    }
}

// Edge table slot of the edge between hex corners a and b.
__device__ __forceinline__ int64_t edge_key(const CubeGrid& g, const HexCorners& h, int a, int b, int& lo,
                                            int& m) {
    lo = min(a, b);
    m = a ^ b;
    return (int64_t)dir_of_bits(m) * g.nv + corner_id(g, h, lo);
}

__global__ void k_cube_vertices(CubeGrid g, double* __restrict__ xyz) {
    const int64_t nxv = g.nx + 1, nyv = g.ny + 1;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < g.nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ix = v % nxv, r = v / nxv;
        const int64_t iy = r % nyv, iz = r / nyv;
        xyz[v] = coord(ix, g.dx);
        xyz[g.n_nodes + v] = coord(iy, g.dy);
        xyz[2 * g.n_nodes + v] = coord(iz, g.dz);
    }
}

// Midpoints staged per warp before a coalesced copy-out: 32 interior hexes create
// 224; a warp on a low boundary face may create more and then writes directly.
constexpr int kMidWarps = 8, kWarpCap = 256;

__global__ void __launch_bounds__(32 * kMidWarps) k_cube_midpoints(CubeGrid g, double* __restrict__ xyz,
                                                                   int32_t* __restrict__ table) {
    __shared__ double stage[3][kMidWarps][kWarpCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t w = (int64_t)blockIdx.x * kMidWarps + warp; w * 32 < g.n_hex; w += (int64_t)gridDim.x * kMidWarps) {
        const int64_t hx = w * 32 + lane;
        const bool active = hx < g.n_hex;
        const int64_t ix = hx % g.nx, r = hx / g.nx;
        const int64_t iy = r % g.ny, iz = r / g.ny;
        const int low[3] = {ix == 0, iy == 0, iz == 0};
        const int64_t first = active ? g.nv + midpoints_before(ix, iy, iz, g.nx, g.ny) : 0;
        const int64_t end = active ? first + owned_count(low[0], low[1], low[2]) : 0;
        const int last = (int)(g.n_hex - 1 - w * 32 < 31 ? g.n_hex - 1 - w * 32 : 31);
        const int64_t base = __shfl_sync(0xffffffffu, first, 0);
        const int total = (int)(__shfl_sync(0xffffffffu, end, last) - base);
        const bool staged = total <= kWarpCap;
        if (active) {
            const HexCorners h = hex_corners(g, ix, iy, iz);
            int64_t id = first;
            unsigned long long seen = 0ull;
            for (int t = 0; t < 6; ++t) {
                int c[4];
                oriented_tet(h, t, c);
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const int a = c[tet_edge(k, 0)], b = c[tet_edge(k, 1)];
                    int lo, m;
                    const int64_t key = edge_key(g, h, a, b, lo, m);
                    const unsigned long long bit = 1ull << (lo * 8 + max(a, b));
                    if (seen & bit) continue;
                    seen |= bit;
                    bool owned = true;
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax)
                        if (!((m >> ax) & 1) && !((lo >> ax) & 1) && !low[ax]) owned = false;
                    if (!owned) continue;
                    table[key] = (int32_t)id;
                    const double px = __dmul_rn(__dadd_rn(h.x(a), h.x(b)), 0.5);
                    const double py = __dmul_rn(__dadd_rn(h.y(a), h.y(b)), 0.5);
                    const double pz = __dmul_rn(__dadd_rn(h.z(a), h.z(b)), 0.5);
                    if (staged) {
                        const int slot = (int)(id - base);
                        stage[0][warp][slot] = px;
                        stage[1][warp][slot] = py;
                        stage[2][warp][slot] = pz;
                    } else {
                        xyz[id] = px;
                        xyz[g.n_nodes + id] = py;
                        xyz[2 * g.n_nodes + id] = pz;
                    }
                    ++id;
                }
            }
        }
        __syncwarp();
        if (staged) {
            for (int i = lane; i < total; i += 32) {
                xyz[base + i] = stage[0][warp][i];
                xyz[g.n_nodes + base + i] = stage[1][warp][i];
                xyz[2 * g.n_nodes + base + i] = stage[2][warp][i];
            }
        }
        __syncwarp();
    }
}

__global__ void k_cube_conn(CubeGrid g, const int32_t* __restrict__ table, int32_t* __restrict__ conn) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < g.n_elem;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t hx = e / 6;
        const int t = (int)(e - 6 * hx);
        const int64_t ix = hx % g.nx, r = hx / g.nx;
        const int64_t iy = r % g.ny, iz = r / g.ny;
        const HexCorners h = hex_corners(g, ix, iy, iz);
        int c[4];
        oriented_tet(h, t, c);
#pragma unroll
        for (int k = 0; k < 4; ++k) conn[k * g.n_elem + e] = (int32_t)corner_id(g, h, c[k]);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            int lo, m;
            const int64_t key = edge_key(g, h, c[tet_edge(k, 0)], c[tet_edge(k, 1)], lo, m);
            conn[(4 + k) * g.n_elem + e] = __ldg(table + key);
        }
    }
}

__global__ void k_soa3_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        aos[3 * i] = soa[i];
        aos[3 * i + 1] = soa[n + i];
        aos[3 * i + 2] = soa[2 * n + i];
    }
}

__global__ void k_conn_to_aos(const int32_t* __restrict__ soa, int32_t* __restrict__ aos, int64_t E) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int l = 0; l < 10; ++l) aos[10 * e + l] = soa[l * E + e];
    }
}

inline unsigned grid_for(const geo_ctx* ctx, int64_t n, int bs) {
    const int64_t cap = (int64_t)ctx->sm_count * 8;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, bs), cap));
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

int geo_mesh_generate_cube(geo_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz,
                           geo_mesh** out) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && out, "ctx/out is NULL");
    GEO_CHECK_ARG(nx > 0 && ny > 0 && nz > 0, "nx, ny and nz must be positive");
    GEO_CHECK_ARG(nx < (int64_t(1) << 20) && ny < (int64_t(1) << 20) && nz < (int64_t(1) << 20),
                  "cube dimension too large");
    int64_t n_nodes = 0, n_elem = 0;
    GEO_CHECK_ARG(geo_generate_cube_size(nx, ny, nz, &n_nodes, &n_elem) == GEO_OK, "invalid cube size");
    GEO_CHECK_ARG(n_nodes < (int64_t(1) << 31) && 10 * n_elem < (int64_t(1) << 31),
                  "mesh too large for 32-bit node ids");
    CubeGrid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.sy = nx + 1;
    g.sz = (nx + 1) * (ny + 1);
    g.nv = g.sz * (nz + 1);
    g.n_nodes = n_nodes;
    g.n_hex = nx * ny * nz;
    g.n_elem = n_elem;
    g.dx = lx / (double)nx;
    g.dy = ly / (double)ny;
    g.dz = lz / (double)nz;
    // the closed-form midpoint count must reproduce the generator's node count
    const int64_t n_mid = plane_count(nx, ny, 1) + (nz - 1) * plane_count(nx, ny, 0);
    if (g.nv + n_mid != n_nodes) fail(GEO_ERR_UNSUPPORTED, "internal: cube midpoint count mismatch");
    auto m = std::make_unique<geo_mesh>();
    m->ctx = ctx;
    m->ref.set(ctx);
    m->n_nodes = n_nodes;
    m->n_elem = n_elem;
    m->xyz.alloc(3 * n_nodes);
    m->conn.alloc(10 * n_elem);
    DevBuf<int32_t> table(7 * g.nv);
    cudaStream_t s = ctx->stream;
    k_cube_vertices<<<grid_for(ctx, g.nv, 256), 256, 0, s>>>(g, m->xyz.p);
    check_launch(ctx, "k_cube_vertices");
    k_cube_midpoints<<<grid_for(ctx, cdiv(g.n_hex, 32), kMidWarps), 32 * kMidWarps, 0, s>>>(g, m->xyz.p, table.p);
    check_launch(ctx, "k_cube_midpoints");
    k_cube_conn<<<grid_for(ctx, g.n_elem, 256), 256, 0, s>>>(g, table.p, m->conn.p);
    check_launch(ctx, "k_cube_conn");
    GEO_CUDA(cudaStreamSynchronize(s));
    *out = m.release();
    GEO_API_END
}

int geo_mesh_size(const geo_mesh* mesh, int64_t* n_nodes, int64_t* n_elem) {
    if (!mesh) return GEO_ERR_INVALID_ARG;
    if (n_nodes) *n_nodes = mesh->n_nodes;
    if (n_elem) *n_elem = mesh->n_elem;
    return GEO_OK;
}

int geo_mesh_download(const geo_mesh* mesh, double* xyz, int32_t* conn) {
    GEO_API_BEGIN(mesh ? mesh->ctx : nullptr)
    GEO_CHECK_ARG(mesh, "mesh is NULL");
    geo_ctx* ctx = mesh->ctx;
    cudaStream_t s = ctx->stream;
    if (xyz) {
        DevBuf<double> tmp;
        double* d = xyz;
        if (!is_device_ptr(xyz)) {
            tmp.alloc(3 * mesh->n_nodes);
            d = tmp.p;
        }
        k_soa3_to_aos<<<grid_for(ctx, mesh->n_nodes, 256), 256, 0, s>>>(mesh->xyz.p, d, mesh->n_nodes);
        check_launch(ctx, "k_soa3_to_aos");
        if (d != xyz) copy_out(xyz, d, 3 * mesh->n_nodes, s);
        GEO_CUDA(cudaStreamSynchronize(s));
    }
    if (conn) {
        DevBuf<int32_t> tmp;
        int32_t* d = conn;
        if (!is_device_ptr(conn)) {
            tmp.alloc(10 * mesh->n_elem);
            d = tmp.p;
        }
        k_conn_to_aos<<<grid_for(ctx, mesh->n_elem, 256), 256, 0, s>>>(mesh->conn.p, d, mesh->n_elem);
        check_launch(ctx, "k_conn_to_aos");
        if (d != conn) copy_out(conn, d, 10 * mesh->n_elem, s);
        GEO_CUDA(cudaStreamSynchronize(s));
    }
    GEO_API_END
}

}  // extern "C"
