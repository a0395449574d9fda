// CPU oracle for the GeoSimulator Tet10 hot path -- TEST INFRASTRUCTURE ONLY.
//
// A line-by-line restatement, in plain C++, of the reference's arithmetic for
// the Tet10 path (msahamed/geo_simulator, Rust). It is the checker for the CUDA
// product and the timed CPU baseline ("reference algorithm restated in C++"):
// the element loop of the `_parallel` assemblers runs under OpenMP in place of
// Rayon, everything else (triplet merge, CSR build, load vectors, Dirichlet
// elimination, Jacobi-CG) is serial, exactly as in the reference.
//
// Third-party arithmetic restated from its published algorithm:
//   * nalgebra 0.33 `Matrix3::try_inverse` / `determinant`: 3x3 adjugate over
//     the cofactor expansion of the first row; `DMatrix::lu`: LU with partial
//     (row) pivoting.  These differ from nalgebra at most in last-bit rounding.
//   * sprs 0.11 `TriMat::to_csr`: rows ascending, columns ascending within a
//     row, duplicates summed in insertion order, explicit zeros kept.  Whether
//     sprs keeps entries whose duplicates sum to exactly 0.0 is not pinned by
//     any reference test; this oracle keeps every structural entry.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>
#include <vector>

namespace {

// ---------------------------------------------------------------- quadrature
// quadrature.rs:13-18 (1 pt), :24-38 (4 pt), :44-59 (5 pt), :65-103 (11 pt)
struct Rule {
    std::vector<std::array<double, 4>> pts;
    std::vector<double> w;
};

Rule rule_1() { return Rule{{{0.25, 0.25, 0.25, 0.25}}, {1.0 / 6.0}}; }

Rule rule_4() {
    const double a = 0.5854101966249685;  // (5 + sqrt 5) / 20
    const double b = 0.1381966011250105;  // (5 - sqrt 5) / 20
    const double w = 1.0 / 24.0;
    return Rule{{{a, b, b, b}, {b, a, b, b}, {b, b, a, b}, {b, b, b, a}}, {w, w, w, w}};
}

Rule rule_5() {
    const double a = 0.25, b = 1.0 / 6.0, c = 0.5;
    return Rule{{{a, a, a, a}, {b, b, b, c}, {b, b, c, b}, {b, c, b, b}, {c, b, b, b}},
                {-2.0 / 15.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0}};
}

Rule rule_11() {
    const double a1 = 0.25, a2 = 0.0714285714285714, b2 = 0.7857142857142857;
    const double a3 = 0.3994035761667992, b3 = 0.1005964238332008;
    Rule r;
    r.pts = {{a1, a1, a1, a1}, {a2, a2, a2, b2}, {a2, a2, b2, a2}, {a2, b2, a2, a2},
             {b2, a2, a2, a2}, {a3, a3, b3, b3}, {a3, b3, a3, b3}, {a3, b3, b3, a3},
             {b3, a3, a3, b3}, {b3, a3, b3, a3}, {b3, b3, a3, a3}};
    r.w = {-0.01315555555555556, 0.007622222222222222, 0.007622222222222222,
           0.007622222222222222, 0.007622222222222222, 0.024888888888888888,
           0.024888888888888888, 0.024888888888888888, 0.024888888888888888,
           0.024888888888888888, 0.024888888888888888};
    return r;
}

// ---------------------------------------------------------------- 3x3 algebra
// Textbook cofactor expansion along the first row (row-major J[3*i + j]).
inline double det3(const double* J) {
    return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
           J[2] * (J[3] * J[7] - J[4] * J[6]);
}

// Inverse through the adjugate; false when the determinant is exactly zero
// (nalgebra's try_inverse returns None only then; basis.rs:247 panics).
inline bool inv3(const double* J, double* Ji) {
    const double d = det3(J);
    if (d == 0.0) return false;
    Ji[0] = (J[4] * J[8] - J[5] * J[7]) / d;
    Ji[1] = (J[2] * J[7] - J[1] * J[8]) / d;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) / d;
    Ji[3] = (J[5] * J[6] - J[3] * J[8]) / d;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) / d;
    Ji[5] = (J[2] * J[3] - J[0] * J[5]) / d;
    Ji[6] = (J[3] * J[7] - J[4] * J[6]) / d;
    Ji[7] = (J[1] * J[6] - J[0] * J[7]) / d;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) / d;
    return true;
}

// ---------------------------------------------------------------- Tet10 basis
// basis.rs:56-73
void shape_functions(const double* L, double* N) {
    const double L0 = L[0], L1 = L[1], L2 = L[2], L3 = L[3];
    N[0] = L0 * (2.0 * L0 - 1.0);
    N[1] = L1 * (2.0 * L1 - 1.0);
    N[2] = L2 * (2.0 * L2 - 1.0);
    N[3] = L3 * (2.0 * L3 - 1.0);
    N[4] = 4.0 * L0 * L1;
    N[5] = 4.0 * L1 * L2;
    N[6] = 4.0 * L2 * L0;
    N[7] = 4.0 * L0 * L3;
    N[8] = 4.0 * L1 * L3;
    N[9] = 4.0 * L2 * L3;
}

// basis.rs:85-110, dN[4*i + m] = dN_i / dL_m
void shape_derivs_bary(const double* L, double* d) {
    const double L0 = L[0], L1 = L[1], L2 = L[2], L3 = L[3];
    const double t[40] = {
        4.0 * L0 - 1.0, 0.0, 0.0, 0.0,
        0.0, 4.0 * L1 - 1.0, 0.0, 0.0,
        0.0, 0.0, 4.0 * L2 - 1.0, 0.0,
        0.0, 0.0, 0.0, 4.0 * L3 - 1.0,
        4.0 * L1, 4.0 * L0, 0.0, 0.0,
        0.0, 4.0 * L2, 4.0 * L1, 0.0,
        4.0 * L2, 0.0, 4.0 * L0, 0.0,
        4.0 * L3, 0.0, 0.0, 4.0 * L0,
        0.0, 4.0 * L3, 0.0, 4.0 * L1,
        0.0, 0.0, 4.0 * L3, 4.0 * L2,
    };
    std::memcpy(d, t, sizeof(t));
}

// basis.rs:196-223, J[3*r + c] = d x_r / d L_{c+1} (L0 eliminated)
void jacobian(const double* L, const double* nodes, double* J) {
    double d[40];
    shape_derivs_bary(L, d);
    for (int k = 0; k < 9; ++k) J[k] = 0.0;
    for (int i = 0; i < 10; ++i) {
        const double x = nodes[3 * i], y = nodes[3 * i + 1], z = nodes[3 * i + 2];
        const double g1 = d[4 * i + 1] - d[4 * i];
        const double g2 = d[4 * i + 2] - d[4 * i];
        const double g3 = d[4 * i + 3] - d[4 * i];
        J[0] += x * g1; J[1] += x * g2; J[2] += x * g3;
        J[3] += y * g1; J[4] += y * g2; J[5] += y * g3;
        J[6] += z * g1; J[7] += z * g2; J[8] += z * g3;
    }
}

// basis.rs:236-276: dN/dx = J^{-T} (dN/dL1 - dN/dL0, ...)
bool shape_derivs_cart(const double* L, const double* nodes, double* dNdx) {
    double d[40], J[9], Ji[9];
    shape_derivs_bary(L, d);
    jacobian(L, nodes, J);
    if (!inv3(J, Ji)) return false;
    for (int i = 0; i < 10; ++i) {
        const double v1 = d[4 * i + 1] - d[4 * i];
        const double v2 = d[4 * i + 2] - d[4 * i];
        const double v3 = d[4 * i + 3] - d[4 * i];
        // (J^{-1})^T v: component a = sum_b Jinv[b][a] v_b
        dNdx[3 * i + 0] = Ji[0] * v1 + Ji[3] * v2 + Ji[6] * v3;
        dNdx[3 * i + 1] = Ji[1] * v1 + Ji[4] * v2 + Ji[7] * v3;
        dNdx[3 * i + 2] = Ji[2] * v1 + Ji[5] * v2 + Ji[8] * v3;
    }
    return true;
}

// ---------------------------------------------------------------- elements
// element.rs:23-61
bool thermal_stiffness(const double* nodes, double k, double* Ke) {
    const Rule q = rule_4();
    for (int i = 0; i < 100; ++i) Ke[i] = 0.0;
    for (size_t p = 0; p < q.pts.size(); ++p) {
        double dNdx[30], J[9];
        if (!shape_derivs_cart(q.pts[p].data(), nodes, dNdx)) return false;
        jacobian(q.pts[p].data(), nodes, J);
        const double w = q.w[p] * std::fabs(det3(J));
        for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j) {
                const double gd = dNdx[3 * i] * dNdx[3 * j] + dNdx[3 * i + 1] * dNdx[3 * j + 1] +
                                  dNdx[3 * i + 2] * dNdx[3 * j + 2];
                Ke[10 * i + j] += k * gd * w;
            }
    }
    return true;
}

// element.rs:74-105 (5-point rule, negative centre weight)
bool thermal_mass(const double* nodes, double rho, double cp, double* Me) {
    const Rule q = rule_5();
    const double rho_cp = rho * cp;
    for (int i = 0; i < 100; ++i) Me[i] = 0.0;
    for (size_t p = 0; p < q.pts.size(); ++p) {
        double N[10], J[9];
        shape_functions(q.pts[p].data(), N);
        jacobian(q.pts[p].data(), nodes, J);
        const double w = q.w[p] * std::fabs(det3(J));
        for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j) Me[10 * i + j] += rho_cp * N[i] * N[j] * w;
    }
    return true;
}

// element.rs:117-140
bool thermal_load(const double* nodes, double Q, double* fe) {
    const Rule q = rule_4();
    for (int i = 0; i < 10; ++i) fe[i] = 0.0;
    for (size_t p = 0; p < q.pts.size(); ++p) {
        double N[10], J[9];
        shape_functions(q.pts[p].data(), N);
        jacobian(q.pts[p].data(), nodes, J);
        const double w = q.w[p] * std::fabs(det3(J));
        for (int i = 0; i < 10; ++i) fe[i] += N[i] * Q * w;
    }
    return true;
}

// mechanics/constitutive.rs:63-102 (factor applied last)
void constitutive(double E, double nu, double* D) {
    const double factor = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double dg = 1.0 - nu, od = nu, sh = (1.0 - 2.0 * nu) / 2.0;
    for (int i = 0; i < 36; ++i) D[i] = 0.0;
    D[0] = dg; D[1] = od; D[2] = od;
    D[6] = od; D[7] = dg; D[8] = od;
    D[12] = od; D[13] = od; D[14] = dg;
    D[21] = sh; D[28] = sh; D[35] = sh;
    for (int i = 0; i < 36; ++i) D[i] = D[i] * factor;
}

// mechanics/strain.rs:38-71, B[30*r + c], rows [xx, yy, zz, xy, yz, zx]
void b_matrix(const double* dNdx, double* B) {
    for (int i = 0; i < 180; ++i) B[i] = 0.0;
    for (int i = 0; i < 10; ++i) {
        const int c = 3 * i;
        const double dx = dNdx[3 * i], dy = dNdx[3 * i + 1], dz = dNdx[3 * i + 2];
        B[0 * 30 + c + 0] = dx;
        B[1 * 30 + c + 1] = dy;
        B[2 * 30 + c + 2] = dz;
        B[3 * 30 + c + 0] = dy;
        B[3 * 30 + c + 1] = dx;
        B[4 * 30 + c + 1] = dz;
        B[4 * 30 + c + 2] = dy;
        B[5 * 30 + c + 2] = dx;
        B[5 * 30 + c + 0] = dz;
    }
}

// mechanics/element.rs:33-65: K_e += w * B^T (D B), per 4-point QP
bool elasticity_stiffness(const double* nodes, double E, double nu, double* Ke) {
    double D[36];
    constitutive(E, nu, D);
    const Rule q = rule_4();
    for (int i = 0; i < 900; ++i) Ke[i] = 0.0;
    for (size_t p = 0; p < q.pts.size(); ++p) {
        double J[9], dNdx[30], B[180], DB[180];
        jacobian(q.pts[p].data(), nodes, J);
        const double dj = det3(J);
        if (!shape_derivs_cart(q.pts[p].data(), nodes, dNdx)) return false;
        b_matrix(dNdx, B);
        const double w = q.w[p] * std::fabs(dj);
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 30; ++c) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += D[6 * r + k] * B[30 * k + c];
                DB[30 * r + c] = s;
            }
        for (int i = 0; i < 30; ++i)
            for (int j = 0; j < 30; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += B[30 * k + i] * DB[30 * k + j];
                Ke[30 * i + j] += w * s;
            }
    }
    return true;
}

// mechanics/body_force.rs:49-84
bool gravity_load(const double* nodes, double rho, const double* g, double* fe) {
    const Rule q = rule_4();
    const double bf[3] = {rho * g[0], rho * g[1], rho * g[2]};
    for (int i = 0; i < 30; ++i) fe[i] = 0.0;
    for (size_t p = 0; p < q.pts.size(); ++p) {
        double N[10], J[9];
        shape_functions(q.pts[p].data(), N);
        jacobian(q.pts[p].data(), nodes, J);
        const double w = q.w[p] * std::fabs(det3(J));
        for (int i = 0; i < 10; ++i) {
            fe[3 * i + 0] += w * N[i] * bf[0];
            fe[3 * i + 1] += w * N[i] * bf[1];
            fe[3 * i + 2] += w * N[i] * bf[2];
        }
    }
    return true;
}

inline void gather_nodes(const double* xyz, const int64_t* conn, int64_t e, double* nodes) {
    for (int i = 0; i < 10; ++i) {
        const int64_t n = conn[10 * e + i];
        nodes[3 * i] = xyz[3 * n];
        nodes[3 * i + 1] = xyz[3 * n + 1];
        nodes[3 * i + 2] = xyz[3 * n + 2];
    }
}

}  // namespace

// ================================================================ CSR object
struct orc_csr {
    int64_t rows = 0, cols = 0;
    std::vector<int64_t> indptr, indices;
    std::vector<double> data;
};

struct orc_mesh {
    std::vector<double> xyz;     // [N][3]
    std::vector<int64_t> conn;   // [E][10]
};

namespace {

// sprs TriMat::to_csr: stable counting sort by row, stable sort by column
// within a row, duplicates summed in insertion order, zeros kept.
orc_csr* triplets_to_csr(int64_t n_rows, int64_t n_cols, const std::vector<int64_t>& r,
                         const std::vector<int64_t>& c, const std::vector<double>& v) {
    const int64_t nt = (int64_t)r.size();
    std::vector<int64_t> cnt(n_rows + 1, 0);
    for (int64_t t = 0; t < nt; ++t) cnt[r[t] + 1]++;
    for (int64_t i = 0; i < n_rows; ++i) cnt[i + 1] += cnt[i];
    std::vector<int64_t> order(nt);
    {
        std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
        for (int64_t t = 0; t < nt; ++t) order[pos[r[t]]++] = t;
    }
    orc_csr* A = new orc_csr;
    A->rows = n_rows;
    A->cols = n_cols;
    A->indptr.assign(n_rows + 1, 0);
    A->indices.reserve(nt);
    A->data.reserve(nt);
    for (int64_t i = 0; i < n_rows; ++i) {
        auto b = order.begin() + cnt[i], e = order.begin() + cnt[i + 1];
        std::stable_sort(b, e, [&](int64_t x, int64_t y) { return c[x] < c[y]; });
        for (auto it = b; it != e;) {
            const int64_t col = c[*it];
            double s = v[*it];
            ++it;
            while (it != e && c[*it] == col) {
                s = s + v[*it];
                ++it;
            }
            A->indices.push_back(col);
            A->data.push_back(s);
        }
        A->indptr[i + 1] = (int64_t)A->indices.size();
    }
    return A;
}

double csr_get(const orc_csr* A, int64_t i, int64_t j, bool* found) {
    auto b = A->indices.begin() + A->indptr[i], e = A->indices.begin() + A->indptr[i + 1];
    auto it = std::lower_bound(b, e, j);
    if (it != e && *it == j) {
        *found = true;
        return A->data[it - A->indices.begin()];
    }
    *found = false;
    return 0.0;
}

// solver.rs:153-155
double norm2(const std::vector<double>& v) {
    double s = 0.0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
}

}  // namespace

extern "C" {

// ================================================================ mesh generator
// mesh_generator_improved.rs:19-169. Vertices first (x fastest, then y, then z);
// hexes in iz/iy/ix order, 6 tets around the v000->v111 diagonal; v2<->v3 swap
// when (v1-v0).((v2-v0)x(v3-v0)) < 0; midpoints first-touch numbered through a
// hash map keyed by the sorted vertex pair, in the order e01 e12 e20 e03 e13 e23.
orc_mesh* orc_generate_cube(int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz) {
    orc_mesh* m = new orc_mesh;
    const double dx = lx / (double)nx, dy = ly / (double)ny, dz = lz / (double)nz;
    auto add_node = [&](double x, double y, double z) {
        m->xyz.push_back(x);
        m->xyz.push_back(y);
        m->xyz.push_back(z);
        return (int64_t)(m->xyz.size() / 3 - 1);
    };
    auto vid = [&](int64_t ix, int64_t iy, int64_t iz) {
        return ix + (nx + 1) * (iy + (ny + 1) * iz);
    };
    for (int64_t iz = 0; iz <= nz; ++iz)
        for (int64_t iy = 0; iy <= ny; ++iy)
            for (int64_t ix = 0; ix <= nx; ++ix)
                add_node((double)ix * dx, (double)iy * dy, (double)iz * dz);

    struct KeyHash {
        size_t operator()(const std::pair<int64_t, int64_t>& k) const {
            return std::hash<int64_t>()(k.first * 0x9E3779B97F4A7C15ull ^ k.second);
        }
    };
    std::unordered_map<std::pair<int64_t, int64_t>, int64_t, KeyHash> cache;
    auto midpoint = [&](int64_t v1, int64_t v2) -> int64_t {
        const auto key = v1 < v2 ? std::make_pair(v1, v2) : std::make_pair(v2, v1);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
        const double* p1 = &m->xyz[3 * v1];
        const double* p2 = &m->xyz[3 * v2];
        const double x = (p1[0] + p2[0]) / 2.0, y = (p1[1] + p2[1]) / 2.0,
                     z = (p1[2] + p2[2]) / 2.0;
        const int64_t id = add_node(x, y, z);
        cache.emplace(key, id);
        return id;
    };
    for (int64_t iz = 0; iz < nz; ++iz)
        for (int64_t iy = 0; iy < ny; ++iy)
            for (int64_t ix = 0; ix < nx; ++ix) {
                const int64_t v000 = vid(ix, iy, iz), v100 = vid(ix + 1, iy, iz),
                              v010 = vid(ix, iy + 1, iz), v110 = vid(ix + 1, iy + 1, iz),
                              v001 = vid(ix, iy, iz + 1), v101 = vid(ix + 1, iy, iz + 1),
                              v011 = vid(ix, iy + 1, iz + 1), v111 = vid(ix + 1, iy + 1, iz + 1);
                const int64_t tets[6][4] = {{v000, v100, v110, v111}, {v000, v100, v111, v101},
                                            {v000, v010, v110, v111}, {v000, v010, v111, v011},
                                            {v000, v001, v111, v101}, {v000, v001, v111, v011}};
                for (int t = 0; t < 6; ++t) {
                    const int64_t v0 = tets[t][0], v1 = tets[t][1];
                    int64_t v2 = tets[t][2], v3 = tets[t][3];
                    const double* p0 = &m->xyz[3 * v0];
                    const double* p1 = &m->xyz[3 * v1];
                    const double* p2 = &m->xyz[3 * v2];
                    const double* p3 = &m->xyz[3 * v3];
                    const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
                    const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
                    const double e3[3] = {p3[0] - p0[0], p3[1] - p0[1], p3[2] - p0[2]};
                    const double cr[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2],
                                          e2[0] * e3[1] - e2[1] * e3[0]};
                    const double det = e1[0] * cr[0] + e1[1] * cr[1] + e1[2] * cr[2];
                    if (det < 0.0) std::swap(v2, v3);
                    const int64_t e01 = midpoint(v0, v1), e12 = midpoint(v1, v2),
                                  e20 = midpoint(v2, v0), e03 = midpoint(v0, v3),
                                  e13 = midpoint(v1, v3), e23 = midpoint(v2, v3);
                    const int64_t el[10] = {v0, v1, v2, v3, e01, e12, e20, e03, e13, e23};
                    m->conn.insert(m->conn.end(), el, el + 10);
                }
            }
    return m;
}

int64_t orc_mesh_num_nodes(const orc_mesh* m) { return (int64_t)(m->xyz.size() / 3); }
int64_t orc_mesh_num_elements(const orc_mesh* m) { return (int64_t)(m->conn.size() / 10); }
void orc_mesh_copy(const orc_mesh* m, double* xyz, int64_t* conn) {
    if (xyz) std::memcpy(xyz, m->xyz.data(), m->xyz.size() * sizeof(double));
    if (conn) std::memcpy(conn, m->conn.data(), m->conn.size() * sizeof(int64_t));
}
void orc_mesh_free(orc_mesh* m) { delete m; }

// ================================================================ basis exports
void orc_shape_functions(const double L[4], double N[10]) { shape_functions(L, N); }
void orc_shape_derivatives_barycentric(const double L[4], double dN[40]) { shape_derivs_bary(L, dN); }
void orc_jacobian(const double L[4], const double nodes[30], double J[9]) { jacobian(L, nodes, J); }
double orc_det3(const double J[9]) { return det3(J); }
int orc_shape_derivatives_cartesian(const double L[4], const double nodes[30], double dNdx[30]) {
    return shape_derivs_cart(L, nodes, dNdx) ? 1 : 0;
}
// basis.rs:352-361
double orc_element_volume(const double nodes[30]) {
    const Rule q = rule_4();
    double v = 0.0;
    for (size_t p = 0; p < q.pts.size(); ++p) {
        double J[9];
        jacobian(q.pts[p].data(), nodes, J);
        v += std::fabs(det3(J)) * q.w[p];
    }
    return v;
}
int orc_quadrature(int rule, double pts[44], double w[11]) {
    Rule r = rule == 1 ? rule_1() : rule == 4 ? rule_4() : rule == 5 ? rule_5() : rule_11();
    for (size_t p = 0; p < r.pts.size(); ++p) {
        for (int m = 0; m < 4; ++m) pts[4 * p + m] = r.pts[p][m];
        w[p] = r.w[p];
    }
    return (int)r.pts.size();
}

int orc_thermal_stiffness(const double nodes[30], double k, double Ke[100]) {
    return thermal_stiffness(nodes, k, Ke) ? 1 : 0;
}
int orc_thermal_mass(const double nodes[30], double rho, double cp, double Me[100]) {
    return thermal_mass(nodes, rho, cp, Me) ? 1 : 0;
}
int orc_thermal_load(const double nodes[30], double Q, double fe[10]) {
    return thermal_load(nodes, Q, fe) ? 1 : 0;
}
void orc_constitutive_matrix(double E, double nu, double D[36]) { constitutive(E, nu, D); }
void orc_b_matrix(const double dNdx[30], double B[180]) { b_matrix(dNdx, B); }
int orc_elasticity_stiffness(const double nodes[30], double E, double nu, double Ke[900]) {
    return elasticity_stiffness(nodes, E, nu, Ke) ? 1 : 0;
}
int orc_gravity_load(const double nodes[30], double rho, const double g[3], double fe[30]) {
    return gravity_load(nodes, rho, g, fe) ? 1 : 0;
}

int orc_thermal_stiffness_all(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn,
                              const double* k_e, double k, double* Ke) {
    (void)n_nodes;
    int ok = 1;
#pragma omp parallel for schedule(static) reduction(&& : ok)
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30];
        gather_nodes(xyz, conn, e, nodes);
        ok = ok && thermal_stiffness(nodes, k_e ? k_e[e] : k, Ke + (size_t)e * 100);
    }
    return ok;
}

// ================================================================ assembly
// assembly.rs:69-117 (parallel) and :22-58 (serial). Rows/cols are node ids.
orc_csr* orc_assemble_thermal_stiffness(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                        const int64_t* conn, const double* k_e, double k,
                                        int parallel) {
    std::vector<double> Ke((size_t)n_elem * 100);
    int ok = 1;
    if (parallel) {
#pragma omp parallel for schedule(static) reduction(&& : ok)
        for (int64_t e = 0; e < n_elem; ++e) {
            double nodes[30];
            gather_nodes(xyz, conn, e, nodes);
            ok = ok && thermal_stiffness(nodes, k_e ? k_e[e] : k, &Ke[(size_t)e * 100]);
        }
    } else {
        for (int64_t e = 0; e < n_elem; ++e) {
            double nodes[30];
            gather_nodes(xyz, conn, e, nodes);
            ok = ok && thermal_stiffness(nodes, k_e ? k_e[e] : k, &Ke[(size_t)e * 100]);
        }
    }
    if (!ok) return nullptr;
    std::vector<int64_t> r, c;
    std::vector<double> v;
    r.reserve((size_t)n_elem * 100);
    c.reserve((size_t)n_elem * 100);
    v.reserve((size_t)n_elem * 100);
    for (int64_t e = 0; e < n_elem; ++e)
        for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j) {
                r.push_back(conn[10 * e + i]);
                c.push_back(conn[10 * e + j]);
                v.push_back(Ke[(size_t)e * 100 + 10 * i + j]);
            }
    return triplets_to_csr(n_nodes, n_nodes, r, c, v);
}

// Same CSR as orc_assemble_thermal_stiffness (sorted columns, duplicates summed
// in element order, structural zeros kept), built row by row under OpenMP
// through a node -> (element, local) map instead of a global triplet sort, so
// that the 128^3 system fits the host's memory and minutes. Used to prepare the
// CPU baseline's input; the arithmetic of every K_e is the reference's.
orc_csr* orc_assemble_thermal_stiffness_rows(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                             const int64_t* conn, const double* k_e, double k) {
    std::vector<double> Ke((size_t)n_elem * 100);
    int ok = 1;
#pragma omp parallel for schedule(static) reduction(&& : ok)
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30];
        gather_nodes(xyz, conn, e, nodes);
        ok = ok && thermal_stiffness(nodes, k_e ? k_e[e] : k, &Ke[(size_t)e * 100]);
    }
    if (!ok) return nullptr;
    std::vector<int64_t> ptr(n_nodes + 1, 0);
    for (int64_t t = 0; t < n_elem * 10; ++t) ptr[conn[t] + 1]++;
    for (int64_t i = 0; i < n_nodes; ++i) ptr[i + 1] += ptr[i];
    std::vector<int64_t> inc(n_elem * 10);
    {
        std::vector<int64_t> cur(ptr.begin(), ptr.end() - 1);
        for (int64_t t = 0; t < n_elem * 10; ++t) inc[cur[conn[t]]++] = t;  // element order
    }
    orc_csr* A = new orc_csr;
    A->rows = A->cols = n_nodes;
    A->indptr.assign(n_nodes + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n_nodes; ++i) {
        std::vector<int64_t> cols;
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int64_t e = inc[p] / 10;
            for (int j = 0; j < 10; ++j) cols.push_back(conn[10 * e + j]);
        }
        std::sort(cols.begin(), cols.end());
        A->indptr[i + 1] = std::unique(cols.begin(), cols.end()) - cols.begin();
    }
    for (int64_t i = 0; i < n_nodes; ++i) A->indptr[i + 1] += A->indptr[i];
    A->indices.resize(A->indptr[n_nodes]);
    A->data.assign(A->indptr[n_nodes], 0.0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n_nodes; ++i) {
        std::vector<int64_t> cols;
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int64_t e = inc[p] / 10;
            for (int j = 0; j < 10; ++j) cols.push_back(conn[10 * e + j]);
        }
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        const int64_t b = A->indptr[i];
        std::copy(cols.begin(), cols.end(), A->indices.begin() + b);
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int64_t e = inc[p] / 10, l = inc[p] % 10;
            for (int j = 0; j < 10; ++j) {
                const int64_t c = conn[10 * e + j];
                const int64_t pos = std::lower_bound(cols.begin(), cols.end(), c) - cols.begin();
                A->data[b + pos] += Ke[(size_t)e * 100 + 10 * l + j];
            }
        }
    }
    return A;
}

// assembly.rs:130-154 (serial element loop)
void orc_assemble_thermal_load(int64_t n_nodes, const double* xyz, int64_t n_elem,
                               const int64_t* conn, double Q, double* f) {
    for (int64_t i = 0; i < n_nodes; ++i) f[i] = 0.0;
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30], fe[10];
        gather_nodes(xyz, conn, e, nodes);
        thermal_load(nodes, Q, fe);
        for (int i = 0; i < 10; ++i) f[conn[10 * e + i]] += fe[i];
    }
}

// assembly.rs:389-437: parallel K_e, then serial triplets with dof = 3*node+comp
orc_csr* orc_assemble_elasticity_stiffness(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                           const int64_t* conn, const double* E_e, double E,
                                           double nu, int parallel) {
    std::vector<double> Ke((size_t)n_elem * 900);
    int ok = 1;
    if (parallel) {
#pragma omp parallel for schedule(static) reduction(&& : ok)
        for (int64_t e = 0; e < n_elem; ++e) {
            double nodes[30];
            gather_nodes(xyz, conn, e, nodes);
            ok = ok && elasticity_stiffness(nodes, E_e ? E_e[e] : E, nu, &Ke[(size_t)e * 900]);
        }
    } else {
        for (int64_t e = 0; e < n_elem; ++e) {
            double nodes[30];
            gather_nodes(xyz, conn, e, nodes);
            ok = ok && elasticity_stiffness(nodes, E_e ? E_e[e] : E, nu, &Ke[(size_t)e * 900]);
        }
    }
    if (!ok) return nullptr;
    std::vector<int64_t> r, c;
    std::vector<double> v;
    r.reserve((size_t)n_elem * 900);
    c.reserve((size_t)n_elem * 900);
    v.reserve((size_t)n_elem * 900);
    for (int64_t e = 0; e < n_elem; ++e)
        for (int i = 0; i < 10; ++i)
            for (int a = 0; a < 3; ++a)
                for (int j = 0; j < 10; ++j)
                    for (int b = 0; b < 3; ++b) {
                        r.push_back(3 * conn[10 * e + i] + a);
                        c.push_back(3 * conn[10 * e + j] + b);
                        v.push_back(Ke[(size_t)e * 900 + 30 * (3 * i + a) + 3 * j + b]);
                    }
    return triplets_to_csr(3 * n_nodes, 3 * n_nodes, r, c, v);
}

// assembly.rs:906-937
void orc_assemble_gravity_load(int64_t n_nodes, const double* xyz, int64_t n_elem,
                               const int64_t* conn, double rho, const double g[3], double* f) {
    for (int64_t i = 0; i < 3 * n_nodes; ++i) f[i] = 0.0;
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30], fe[30];
        gather_nodes(xyz, conn, e, nodes);
        gravity_load(nodes, rho, g, fe);
        for (int i = 0; i < 10; ++i)
            for (int a = 0; a < 3; ++a) f[3 * conn[10 * e + i] + a] += fe[3 * i + a];
    }
}

// assembly.rs:184-193
double orc_char_diag(const orc_csr* K) {
    double max_diag = 1.0;
    for (int64_t i = 0; i < K->rows; ++i)
        for (int64_t p = K->indptr[i]; p < K->indptr[i + 1]; ++p)
            if (K->indices[p] == i) {
                const double a = std::fabs(K->data[p]);
                if (a > max_diag) max_diag = a;
            }
    return max_diag;
}

// assembly.rs:168-230
orc_csr* orc_apply_dirichlet_bcs(const orc_csr* K, const double* f, const uint8_t* mask,
                                 const double* g, double* f_out) {
    const int64_t n = K->rows;
    const double cd = orc_char_diag(K);
    for (int64_t i = 0; i < n; ++i) f_out[i] = f[i];
    for (int64_t i = 0; i < n; ++i) {
        if (mask[i]) continue;
        for (int64_t p = K->indptr[i]; p < K->indptr[i + 1]; ++p) {
            const int64_t j = K->indices[p];
            if (mask[j]) f_out[i] -= K->data[p] * g[j];
        }
    }
    std::vector<int64_t> r, c;
    std::vector<double> v;
    for (int64_t i = 0; i < n; ++i) {
        if (mask[i]) {
            r.push_back(i);
            c.push_back(i);
            v.push_back(cd);
            f_out[i] = g[i] * cd;
        } else {
            for (int64_t p = K->indptr[i]; p < K->indptr[i + 1]; ++p) {
                const int64_t j = K->indices[p];
                if (!mask[j]) {
                    r.push_back(i);
                    c.push_back(j);
                    v.push_back(K->data[p]);
                }
            }
        }
    }
    return triplets_to_csr(n, K->cols, r, c, v);
}

// assembly.rs:168-230 with the same results as orc_apply_dirichlet_bcs (each
// (row, col) occurs once, so the triplet merge is a per-row copy), row-parallel.
orc_csr* orc_apply_dirichlet_bcs_rows(const orc_csr* K, const double* f, const uint8_t* mask, const double* g,
                                      double* f_out) {
    const int64_t n = K->rows;
    const double cd = orc_char_diag(K);
    orc_csr* B = new orc_csr;
    B->rows = n;
    B->cols = K->cols;
    B->indptr.assign(n + 1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        if (mask[i]) {
            B->indptr[i + 1] = 1;
            f_out[i] = g[i] * cd;
            continue;
        }
        double s = f[i];
        int64_t c = 0;
        for (int64_t p = K->indptr[i]; p < K->indptr[i + 1]; ++p) {
            const int64_t j = K->indices[p];
            if (mask[j]) s -= K->data[p] * g[j];
            else ++c;
        }
        f_out[i] = s;
        B->indptr[i + 1] = c;
    }
    for (int64_t i = 0; i < n; ++i) B->indptr[i + 1] += B->indptr[i];
    B->indices.resize(B->indptr[n]);
    B->data.resize(B->indptr[n]);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int64_t o = B->indptr[i];
        if (mask[i]) {
            B->indices[o] = i;
            B->data[o] = cd;
            continue;
        }
        for (int64_t p = K->indptr[i]; p < K->indptr[i + 1]; ++p) {
            const int64_t j = K->indices[p];
            if (!mask[j]) {
                B->indices[o] = j;
                B->data[o] = K->data[p];
                ++o;
            }
        }
    }
    return B;
}

orc_csr* orc_csr_from_triplets(int64_t n_rows, int64_t n_cols, int64_t n_trip, const int64_t* rows,
                               const int64_t* cols, const double* vals) {
    std::vector<int64_t> r(rows, rows + n_trip), c(cols, cols + n_trip);
    std::vector<double> v(vals, vals + n_trip);
    return triplets_to_csr(n_rows, n_cols, r, c, v);
}
// Copies an existing CSR (already sorted and merged) into an oracle handle.
orc_csr* orc_csr_wrap(int64_t n_rows, int64_t n_cols, const int64_t* indptr, const int32_t* indices,
                      const double* data) {
    orc_csr* A = new orc_csr;
    A->rows = n_rows;
    A->cols = n_cols;
    const int64_t nnz = indptr[n_rows];
    A->indptr.assign(indptr, indptr + n_rows + 1);
    A->indices.resize(nnz);
    for (int64_t p = 0; p < nnz; ++p) A->indices[p] = indices[p];
    A->data.assign(data, data + nnz);
    return A;
}
int64_t orc_csr_rows(const orc_csr* A) { return A->rows; }
int64_t orc_csr_nnz(const orc_csr* A) { return (int64_t)A->indices.size(); }
void orc_csr_copy(const orc_csr* A, int64_t* indptr, int64_t* indices, double* data) {
    if (indptr) std::memcpy(indptr, A->indptr.data(), A->indptr.size() * sizeof(int64_t));
    if (indices) std::memcpy(indices, A->indices.data(), A->indices.size() * sizeof(int64_t));
    if (data) std::memcpy(data, A->data.data(), A->data.size() * sizeof(double));
}
// solver.rs:61-73
void orc_csr_apply(const orc_csr* A, const double* x, double* y) {
    for (int64_t i = 0; i < A->rows; ++i) {
        double s = 0.0;
        for (int64_t p = A->indptr[i]; p < A->indptr[i + 1]; ++p) s += A->data[p] * x[A->indices[p]];
        y[i] = s;
    }
}
void orc_csr_free(orc_csr* A) { delete A; }

// ================================================================ solvers
// iterative.rs:46-131 with preconditioner.rs:37-72 (Jacobi / identity)
void orc_cg_solve(const orc_csr* A, const double* b, int64_t max_iterations, double tolerance,
                  double abs_tolerance, int use_preconditioner, double* x_out, orc_stats* st) {
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t n = A->rows;
    std::vector<double> diag_inv(n, 1.0);
    if (use_preconditioner) {
        for (int64_t i = 0; i < n; ++i) {
            bool found;
            const double v = csr_get(A, i, i, &found);
            if (found && std::fabs(v) > 1e-14) diag_inv[i] = 1.0 / v;
        }
    }
    auto precond = [&](const std::vector<double>& r) {
        std::vector<double> z(n);
        for (int64_t i = 0; i < n; ++i) z[i] = r[i] * diag_inv[i];
        return z;
    };
    auto elapsed = [&]() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    };
    std::vector<double> bv(b, b + n);
    const double b_norm = norm2(bv);
    if (b_norm < 1e-25) {
        for (int64_t i = 0; i < n; ++i) x_out[i] = 0.0;
        *st = orc_stats{0, 0.0, 0.0, 1, elapsed()};
        return;
    }
    std::vector<double> x(n, 0.0), r = bv, ap(n);
    std::vector<double> z = precond(r);
    std::vector<double> p = z;
    double rz = 0.0;
    for (int64_t i = 0; i < n; ++i) rz += r[i] * z[i];
    int64_t it = 0;
    bool converged = false;
    double final_res = b_norm;
    while (it < max_iterations) {
        orc_csr_apply(A, p.data(), ap.data());
        double p_ap = 0.0;
        for (int64_t i = 0; i < n; ++i) p_ap += p[i] * ap[i];
        if (std::fabs(p_ap) < 1e-30) break;
        const double alpha = rz / p_ap;
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * ap[i];
        }
        const double r_norm = norm2(r);
        final_res = r_norm;
        if (r_norm < tolerance * b_norm || r_norm < abs_tolerance) {
            converged = true;
            break;
        }
        z = precond(r);
        double rz_new = 0.0;
        for (int64_t i = 0; i < n; ++i) rz_new += r[i] * z[i];
        const double beta = rz_new / rz;
        rz = rz_new;
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        it += 1;
    }
    for (int64_t i = 0; i < n; ++i) x_out[i] = x[i];
    *st = orc_stats{it, final_res, b_norm > 1e-20 ? final_res / b_norm : 0.0, converged ? 1 : 0,
                    elapsed()};
}

// Jacobi (preconditioner.rs:37-62) or identity inverse diagonal
static std::vector<double> jacobi_inverse(const orc_csr* A, int use_preconditioner) {
    std::vector<double> d((size_t)A->rows, 1.0);
    if (use_preconditioner)
        for (int64_t i = 0; i < A->rows; ++i) {
            bool found;
            const double v = csr_get(A, i, i, &found);
            if (found && std::fabs(v) > 1e-14) d[(size_t)i] = 1.0 / v;
        }
    return d;
}

static double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// BiCGSTAB::solve_with_operator_internal (iterative.rs:177-278), right-preconditioned
void orc_bicgstab_solve(const orc_csr* A, const double* b, int64_t max_iterations, double tolerance,
                        double abs_tolerance, int use_preconditioner, double* x_out, orc_stats* st) {
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t n = A->rows;
    const std::vector<double> dinv = jacobi_inverse(A, use_preconditioner);
    auto elapsed = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    std::vector<double> bv(b, b + n);
    const double b_norm = norm2(bv);
    if (b_norm < 1e-25) {
        for (int64_t i = 0; i < n; ++i) x_out[i] = 0.0;
        *st = orc_stats{0, 0.0, 0.0, 1, elapsed()};
        return;
    }
    std::vector<double> x(n, 0.0), r = bv, r_hat = bv, v(n, 0.0), p(n, 0.0), p_hat(n), s(n), s_hat(n), t(n);
    double rho = 1.0, alpha = 1.0, omega = 1.0, final_res = b_norm;
    int64_t total = 0;
    bool converged = false;
    while (total < max_iterations) {
        const double rho_prev = rho;
        rho = dot(r_hat, r);
        if (std::fabs(rho) < 1e-40) break;
        if (total == 0) {
            p = r;
        } else {
            const double beta = (rho / rho_prev) * (alpha / omega);
            for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        }
        for (int64_t i = 0; i < n; ++i) p_hat[i] = p[i] * dinv[i];
        orc_csr_apply(A, p_hat.data(), v.data());
        const double rhat_v = dot(r_hat, v);
        if (std::fabs(rhat_v) < 1e-40) break;
        alpha = rho / rhat_v;
        for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        const double s_norm = norm2(s);
        if (s_norm < tolerance * b_norm || s_norm < abs_tolerance) {
            for (int64_t i = 0; i < n; ++i) x[i] += alpha * p_hat[i];
            final_res = s_norm;
            converged = true;
            break;
        }
        for (int64_t i = 0; i < n; ++i) s_hat[i] = s[i] * dinv[i];
        orc_csr_apply(A, s_hat.data(), t.data());
        const double t_t = dot(t, t), t_s = dot(t, s);
        if (std::fabs(t_t) < 1e-40) break;
        omega = t_s / t_t;
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p_hat[i] + omega * s_hat[i];
            r[i] = s[i] - omega * t[i];
        }
        final_res = norm2(r);
        total += 1;
        if (final_res < tolerance * b_norm || final_res < abs_tolerance) {
            converged = true;
            break;
        }
        if (std::fabs(omega) < 1e-40) break;
    }
    for (int64_t i = 0; i < n; ++i) x_out[i] = x[i];
    *st = orc_stats{total, final_res, final_res / b_norm, converged ? 1 : 0, elapsed()};
}

// GMRES::solve_with_operator_internal (iterative.rs:333-456): restarted, right-
// preconditioned, modified Gram-Schmidt, Givens rotations (givens_rotation, :458-467)
void orc_gmres_solve(const orc_csr* A, const double* b, int64_t max_iterations, int64_t restart, double tolerance,
                     double abs_tolerance, int use_preconditioner, double* x_out, orc_stats* st) {
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t n = A->rows;
    const std::vector<double> dinv = jacobi_inverse(A, use_preconditioner);
    auto elapsed = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    std::vector<double> bv(b, b + n);
    const double b_norm = norm2(bv);
    if (b_norm < 1e-25) {
        for (int64_t i = 0; i < n; ++i) x_out[i] = 0.0;
        *st = orc_stats{0, 0.0, 0.0, 1, elapsed()};
        return;
    }
    auto givens = [](double a, double bb, double& c, double& s, double& rho) {
        if (std::fabs(bb) < 1e-40) {
            c = 1.0;
            s = 0.0;
            rho = a;
        } else if (std::fabs(bb) > std::fabs(a)) {
            const double tau = a / bb;
            s = 1.0 / std::sqrt(1.0 + tau * tau);
            c = s * tau;
            rho = bb * std::sqrt(1.0 + tau * tau);
        } else {
            const double tau = bb / a;
            c = 1.0 / std::sqrt(1.0 + tau * tau);
            s = c * tau;
            rho = a * std::sqrt(1.0 + tau * tau);
        }
    };
    std::vector<double> x(n, 0.0), r(n), w(n), z(n);
    int64_t total = 0;
    bool converged = false;
    double final_res = b_norm;
    const int64_t m = restart;
    while (total < max_iterations) {
        orc_csr_apply(A, x.data(), r.data());  // r = b - A x
        for (int64_t i = 0; i < n; ++i) r[i] = bv[i] - r[i];
        const double r_norm = norm2(r);
        final_res = r_norm;
        if (r_norm < tolerance * b_norm || r_norm < abs_tolerance) {
            converged = true;
            break;
        }
        std::vector<std::vector<double>> v((size_t)m + 1, std::vector<double>(n, 0.0));
        std::vector<std::vector<double>> h((size_t)m + 1, std::vector<double>((size_t)m, 0.0));
        for (int64_t i = 0; i < n; ++i) v[0][i] = r[i] / r_norm;
        std::vector<double> g((size_t)m + 1, 0.0), cs((size_t)m, 0.0), sn((size_t)m, 0.0);
        g[0] = r_norm;
        int64_t k = 0;
        for (int64_t j = 0; j < m; ++j) {
            if (total >= max_iterations) break;
            for (int64_t i = 0; i < n; ++i) z[i] = v[j][i] * dinv[i];
            orc_csr_apply(A, z.data(), w.data());
            for (int64_t i = 0; i <= j; ++i) {
                h[i][j] = dot(v[i], w);
                for (int64_t l = 0; l < n; ++l) w[l] -= h[i][j] * v[i][l];
            }
            h[j + 1][j] = norm2(w);
            if (std::fabs(h[j + 1][j]) > 1e-40)
                for (int64_t l = 0; l < n; ++l) v[j + 1][l] = w[l] / h[j + 1][j];
            for (int64_t i = 0; i < j; ++i) {
                const double temp = cs[i] * h[i][j] + sn[i] * h[i + 1][j];
                h[i + 1][j] = -sn[i] * h[i][j] + cs[i] * h[i + 1][j];
                h[i][j] = temp;
            }
            double c, s, rho;
            givens(h[j][j], h[j + 1][j], c, s, rho);
            cs[j] = c;
            sn[j] = s;
            h[j][j] = rho;
            h[j + 1][j] = 0.0;
            const double temp = cs[j] * g[j];
            g[j + 1] = -sn[j] * g[j];
            g[j] = temp;
            k = j + 1;
            total += 1;
            final_res = std::fabs(g[k]);
            if (final_res < tolerance * b_norm || final_res < abs_tolerance) break;
        }
        std::vector<double> y((size_t)k, 0.0);
        for (int64_t i = k - 1; i >= 0; --i) {
            double sum = 0.0;
            for (int64_t j = i + 1; j < k; ++j) sum += h[i][j] * y[j];
            if (std::fabs(h[i][i]) < 1e-40) break;
            y[i] = (g[i] - sum) / h[i][i];
        }
        std::vector<double> dy(n, 0.0);
        for (int64_t j = 0; j < k; ++j)
            for (int64_t i = 0; i < n; ++i) dy[i] += v[j][i] * y[j];
        for (int64_t i = 0; i < n; ++i) x[i] += dy[i] * dinv[i];
        if (final_res < tolerance * b_norm || final_res < abs_tolerance) {
            converged = true;
            break;
        }
    }
    for (int64_t i = 0; i < n; ++i) x_out[i] = x[i];
    *st = orc_stats{total, final_res, final_res / b_norm, converged ? 1 : 0, elapsed()};
}

// direct.rs:28-73: dense LU with partial pivoting; converged <=> rel-res < 1e-8
int orc_lu_solve(const orc_csr* A, const double* b, double* x, orc_stats* st) {
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t n = A->rows;
    std::vector<double> M((size_t)n * n, 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t p = A->indptr[i]; p < A->indptr[i + 1]; ++p) M[(size_t)i * n + A->indices[p]] = A->data[p];
    std::vector<int64_t> piv(n);
    std::iota(piv.begin(), piv.end(), 0);
    for (int64_t k = 0; k < n; ++k) {
        int64_t pr = k;
        double best = std::fabs(M[(size_t)k * n + k]);
        for (int64_t i = k + 1; i < n; ++i)
            if (std::fabs(M[(size_t)i * n + k]) > best) {
                best = std::fabs(M[(size_t)i * n + k]);
                pr = i;
            }
        if (best == 0.0) return 0;
        if (pr != k) {
            for (int64_t j = 0; j < n; ++j) std::swap(M[(size_t)k * n + j], M[(size_t)pr * n + j]);
            std::swap(piv[k], piv[pr]);
        }
        const double d = M[(size_t)k * n + k];
        for (int64_t i = k + 1; i < n; ++i) {
            const double l = M[(size_t)i * n + k] / d;
            M[(size_t)i * n + k] = l;
            if (l == 0.0) continue;
            double* ri = &M[(size_t)i * n];
            const double* rk = &M[(size_t)k * n];
            for (int64_t j = k + 1; j < n; ++j) ri[j] -= l * rk[j];
        }
    }
    std::vector<double> y(n);
    for (int64_t i = 0; i < n; ++i) {
        double s = b[piv[i]];
        for (int64_t j = 0; j < i; ++j) s -= M[(size_t)i * n + j] * y[j];
        y[i] = s;
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int64_t j = i + 1; j < n; ++j) s -= M[(size_t)i * n + j] * x[j];
        x[i] = s / M[(size_t)i * n + i];
    }
    const double solve_time =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    // solver.rs:139-175
    std::vector<double> ax(n), r(n);
    orc_csr_apply(A, x, ax.data());
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
    const double rn = norm2(r);
    const double bn = norm2(std::vector<double>(b, b + n));
    const double rel = bn < 1e-14 ? rn : rn / bn;
    *st = orc_stats{0, rn, rel, rel < 1e-8 ? 1 : 0, solve_time};
    return 1;
}

// ================================================================ adjoint checker
// g_e = -lambda_e^T K_e(k_e) u_e: derivative of J with respect to ln k_e for the
// Dirichlet-eliminated system when lambda solves K_bc lambda = dJ/du with
// lambda = 0 on Dirichlet DOFs (K_e is linear in k_e). No reference counterpart.
void orc_thermal_element_gradient(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                  const int64_t* conn, const double* k_e, const double* u,
                                  const double* lam, double* g) {
    (void)n_nodes;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30], Ke[100];
        gather_nodes(xyz, conn, e, nodes);
        thermal_stiffness(nodes, k_e[e], Ke);
        double s = 0.0;
        for (int i = 0; i < 10; ++i) {
            double t = 0.0;
            for (int j = 0; j < 10; ++j) t += Ke[10 * i + j] * u[conn[10 * e + j]];
            s += lam[conn[10 * e + i]] * t;
        }
        g[e] = -s;
    }
}

void orc_elasticity_element_gradient(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                     const int64_t* conn, const double* E_e, double nu,
                                     const double* u, const double* lam, double* g) {
    (void)n_nodes;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30];
        std::vector<double> Ke(900);
        gather_nodes(xyz, conn, e, nodes);
        elasticity_stiffness(nodes, E_e[e], nu, Ke.data());
        double s = 0.0;
        for (int i = 0; i < 30; ++i) {
            double t = 0.0;
            for (int j = 0; j < 30; ++j) t += Ke[30 * i + j] * u[3 * conn[10 * e + j / 3] + j % 3];
            s += lam[3 * conn[10 * e + i / 3] + i % 3] * t;
        }
        g[e] = -s;
    }
}

}  // extern "C"

// ---------------------------------------------------------------- Neumann (flux) boundary
// Tet10Face::from_element_face, fem/boundary.rs:89-130: 3 vertices then the 3
// edge midpoints of local face f (face f is opposite vertex f).
static const int kFace[4][6] = {
    {1, 2, 3, 5, 9, 8},
    {0, 2, 3, 6, 9, 7},
    {0, 1, 3, 4, 8, 7},
    {0, 1, 2, 4, 5, 6},
};

void orc_face_nodes(const int64_t elem[10], int local_face, int64_t out[6]) {
    for (int i = 0; i < 6; ++i) out[i] = elem[kFace[local_face][i]];
}

// 6-node triangle shape functions and derivatives in area coordinates (L1, L2),
// L3 = 1 - L1 - L2, boundary.rs:145-167 / :206-228.
static void tri6(double l1, double l2, double N[6], double d[6][2]) {
    const double l3 = 1.0 - l1 - l2;
    N[0] = l1 * (2.0 * l1 - 1.0);
    N[1] = l2 * (2.0 * l2 - 1.0);
    N[2] = l3 * (2.0 * l3 - 1.0);
    N[3] = 4.0 * l1 * l2;
    N[4] = 4.0 * l2 * l3;
    N[5] = 4.0 * l3 * l1;
    d[0][0] = 4.0 * l1 - 1.0;  d[0][1] = 0.0;
    d[1][0] = 0.0;             d[1][1] = 4.0 * l2 - 1.0;
    d[2][0] = -4.0 * l3 + 1.0; d[2][1] = -4.0 * l3 + 1.0;
    d[3][0] = 4.0 * l2;        d[3][1] = 4.0 * l1;
    d[4][0] = -4.0 * l2;       d[4][1] = 4.0 * (l3 - l2);
    d[5][0] = 4.0 * (l3 - l1); d[5][1] = -4.0 * l1;
}

// 3-point triangle rule, boundary.rs:172-176 / :232-236 (weights sum to 1/2)
static const double kTriQ[3][3] = {
    {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0},
    {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
    {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0},
};

// |dx/dL1 x dx/dL2| at (l1, l2); coords [6][3]
static double tri6_detj(const double* c, const double d[6][2]) {
    double a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
    for (int i = 0; i < 6; ++i)
        for (int k = 0; k < 3; ++k) {
            a[k] += c[3 * i + k] * d[i][0];
            b[k] += c[3 * i + k] * d[i][1];
        }
    const double x = a[1] * b[2] - a[2] * b[1], y = a[2] * b[0] - a[0] * b[2], z = a[0] * b[1] - a[1] * b[0];
    return std::sqrt(x * x + y * y + z * z);
}

// Tet10Face::area, boundary.rs:136-196
double orc_face_area(const double coords[18]) {
    double area = 0.0;
    for (int q = 0; q < 3; ++q) {
        double N[6], d[6][2];
        tri6(kTriQ[q][0], kTriQ[q][1], N, d);
        area += kTriQ[q][2] * tri6_detj(coords, d);
    }
    return area;
}

// Tet10Face::integrate_flux, boundary.rs:202-266: f_i = sum_q w_q N_i flux |det J|
void orc_face_flux(const double coords[18], double flux, double f[6]) {
    for (int i = 0; i < 6; ++i) f[i] = 0.0;
    for (int q = 0; q < 3; ++q) {
        double N[6], d[6][2];
        tri6(kTriQ[q][0], kTriQ[q][1], N, d);
        const double dj = tri6_detj(coords, d);
        for (int i = 0; i < 6; ++i) f[i] += kTriQ[q][2] * N[i] * flux * dj;
    }
}

// Assembler::find_boundary_faces, assembly.rs:287-309: faces whose 6 nodes all
// satisfy the condition (node_mask), element-major then local face. Returns the count.
int64_t orc_find_boundary_faces(int64_t n_elem, const int64_t* conn, const uint8_t* node_mask, int64_t* faces) {
    int64_t n = 0;
    for (int64_t e = 0; e < n_elem; ++e)
        for (int f = 0; f < 4; ++f) {
            bool all = true;
            for (int i = 0; i < 6 && all; ++i) all = node_mask[conn[10 * e + kFace[f][i]]] != 0;
            if (all) {
                faces[2 * n] = e;
                faces[2 * n + 1] = f;
                ++n;
            }
        }
    return n;
}

// Assembler::apply_neumann_bcs, assembly.rs:248-274: f[node] += face flux
// contributions, faces in the given order.
void orc_apply_neumann_bcs(const double* xyz, const int64_t* conn, int64_t n_faces, const int64_t* faces,
                           const double* flux, double* f) {
    for (int64_t k = 0; k < n_faces; ++k) {
        int64_t nodes[6];
        orc_face_nodes(conn + 10 * faces[2 * k], (int)faces[2 * k + 1], nodes);
        double c[18], fe[6];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 3; ++j) c[3 * i + j] = xyz[3 * nodes[i] + j];
        orc_face_flux(c, flux[k], fe);
        for (int i = 0; i < 6; ++i) f[nodes[i]] += fe[i];
    }
}

// ---------------------------------------------------------------- Maxwell viscoelasticity
// ElasticityElement::maxwell_viscoelastic (mechanics/element.rs:257-296), history part:
// f_e = -sum_q w_q |det J_q| B_q^T sigma_n (4-point rule, isoparametric B); the
// stiffness part is the elastic K_e (elasticity_stiffness). Scattered as in
// Assembler::assemble_maxwell_viscoelastic_parallel (assembly.rs:959-1020):
// element order, node i, component c.
int orc_maxwell_history_force(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn,
                              const double* stress, double* f) {
    for (int64_t i = 0; i < 3 * n_nodes; ++i) f[i] = 0.0;
    const Rule q = rule_4();
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30], fe[30] = {0};
        gather_nodes(xyz, conn, e, nodes);
        const double* sg = stress + 6 * e;
        for (size_t p = 0; p < q.pts.size(); ++p) {
            double J[9], dNdx[30], B[180];
            jacobian(q.pts[p].data(), nodes, J);
            const double w = q.w[p] * std::fabs(det3(J));
            if (!shape_derivs_cart(q.pts[p].data(), nodes, dNdx)) return 1;
            b_matrix(dNdx, B);
            for (int c = 0; c < 30; ++c) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += B[30 * k + c] * sg[k];
                fe[c] -= w * s;
            }
        }
        for (int i = 0; i < 10; ++i)
            for (int c = 0; c < 3; ++c) f[3 * conn[10 * e + i] + c] += fe[3 * i + c];
    }
    return 0;
}

// update_stresses_maxwell (mechanics/stress_update.rs:39-143): strain increment
// averaged over the 4 points, elastic predictor with lambda = K - 2G/3,
// deviatoric part relaxed by 1 / (1 + dt / tau_M), tau_M = mu / G.
int orc_update_stresses_maxwell(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, double E,
                                double nu, double mu, const double* u_n, const double* u_next, double dt,
                                const double* stress_n, double* stress_next) {
    (void)n_nodes;
    const double G = E / (2.0 * (1.0 + nu));
    const double tau = mu / G;
    const double factor = 1.0 / (1.0 + dt / tau);
    const double Kb = E / (3.0 * (1.0 - 2.0 * nu));
    const double lam = Kb - 2.0 * G / 3.0;
    const Rule q = rule_4();
    for (int64_t e = 0; e < n_elem; ++e) {
        double nodes[30], du[30], de[6] = {0, 0, 0, 0, 0, 0};
        gather_nodes(xyz, conn, e, nodes);
        for (int i = 0; i < 10; ++i)
            for (int c = 0; c < 3; ++c) {
                const int64_t g = 3 * conn[10 * e + i] + c;
                du[3 * i + c] = u_next[g] - u_n[g];
            }
        for (size_t p = 0; p < q.pts.size(); ++p) {
            double dNdx[30], B[180];
            if (!shape_derivs_cart(q.pts[p].data(), nodes, dNdx)) return 1;
            b_matrix(dNdx, B);
            for (int k = 0; k < 6; ++k) {
                double s = 0.0;
                for (int c = 0; c < 30; ++c) s += B[30 * k + c] * du[c];
                de[k] += s;
            }
        }
        for (int k = 0; k < 6; ++k) de[k] /= (double)q.pts.size();
        const double* sn = stress_n + 6 * e;
        const double tr = de[0] + de[1] + de[2];
        double st[6] = {sn[0] + lam * tr + 2.0 * G * de[0], sn[1] + lam * tr + 2.0 * G * de[1],
                        sn[2] + lam * tr + 2.0 * G * de[2], sn[3] + G * de[3],
                        sn[4] + G * de[4],                  sn[5] + G * de[5]};
        const double p = (st[0] + st[1] + st[2]) / 3.0;
        double* o = stress_next + 6 * e;
        o[0] = (st[0] - p) * factor + p;
        o[1] = (st[1] - p) * factor + p;
        o[2] = (st[2] - p) * factor + p;
        o[3] = st[3] * factor;
        o[4] = st[4] * factor;
        o[5] = st[5] * factor;
    }
    return 0;
}
