// C++ host tests of geofem.hpp on the GPU, written the way the reference's own
// Rust tests and benchmarks use its API:
//   thermal 1D profile      benchmarks/thermal_1d_improved_mesh.rs:9-66
//   2x2 CG                  src/linalg/iterative.rs:490-504
//   diagonal Jacobi         src/linalg/preconditioner.rs:212-230
//   elasticity patch test   benchmarks/elasticity_patch_test.rs:14-107
//   panics -> errors        src/fem/basis.rs:247, src/fem/assembly.rs:394
// plus the matrix-free mixed-precision solve and the adjoint against central
// finite differences (no reference counterpart). Prints one line per test and
// exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "geofem.hpp"

using namespace geofem;

namespace {

int g_failures = 0;

void expect(bool ok, const std::string& what) {
    std::printf("%s %s\n", ok ? "ok  " : "FAIL", what.c_str());
    if (!ok) ++g_failures;
}

double max_abs_diff(const std::vector<double>& a, const std::vector<double>& b) {
    double m = 0;
    for (size_t i = 0; i < a.size(); ++i) m = std::fmax(m, std::fabs(a[i] - b[i]));
    return m;
}

std::string sci(double v) {
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%.2e", v);
    return buf;
}

double rel_l2(const std::vector<double>& a, const std::vector<double>& b) {
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        num += (a[i] - b[i]) * (a[i] - b[i]);
        den += b[i] * b[i];
    }
    return std::sqrt(num / std::fmax(den, 1e-300));
}

// T(z) = T_b + (T_t - T_b) z / L + Q / (2k) z (L - z)
double analytic(double z, double lz, double tb, double tt, double k, double q) {
    return tb + (tt - tb) * (z / lz) + (q / (2.0 * k)) * z * (lz - z);
}

DofManager thermal_dofs(const Mesh& mesh, double lz, double tb, double tt) {
    DofManager d(mesh.num_nodes(), 1);
    for (size_t i = 0; i < mesh.num_nodes(); ++i) {
        const double z = mesh.nodes[i][2];
        if (std::fabs(z) < 1.0) d.set_dirichlet_node(i, tb);
        else if (std::fabs(z - lz) < 1.0) d.set_dirichlet_node(i, tt);
    }
    return d;
}

void thermal_profile() {
    const double lx = 1000, ly = 1000, lz = 600, tb = 1280, tt = 0, k = 3.0, q = 1e-6;
    for (int n : {2, 4, 6}) {
        Mesh mesh = ImprovedMeshGenerator::generate_cube(n, n, n, lx, ly, lz);
        DofManager dofs = thermal_dofs(mesh, lz, tb, tt);
        CsMat K = Assembler::assemble_thermal_stiffness_parallel(mesh, dofs, k);
        std::vector<double> f = Assembler::assemble_thermal_load(mesh, dofs, q);
        auto kb = Assembler::apply_dirichlet_bcs(K, f, dofs);
        auto sol = ConjugateGradient().with_max_iterations(1000).with_tolerance(1e-10).solve(kb.first, kb.second);
        double err = 0;
        for (size_t i = 0; i < mesh.num_nodes(); ++i)
            err = std::fmax(err, std::fabs(sol.first[i] - analytic(mesh.nodes[i][2], lz, tb, tt, k, q)));
        expect(sol.second.converged && err < 1e-6 * tb,
               "thermal 1D profile " + std::to_string(n) + "^3: max |T - T_exact| = " + sci(err) +
                   ", " + std::to_string(sol.second.iterations) + " iterations");
        // the same system matrix-free, FP64 and mixed precision
        ThermalOperator op(mesh, dofs, k);
        for (Precision p : {Precision::FP64, Precision::Mixed}) {
            auto mf = op.solve(kb.second, ConjugateGradient().with_tolerance(1e-10).with_precision(p));
            const double e = rel_l2(mf.first, sol.first);
            expect(mf.second.converged && e < 1e-8,
                   std::string("matrix-free ") + (p == Precision::FP64 ? "fp64" : "mixed") + " vs CSR " +
                       std::to_string(n) + "^3: rel L2 " + sci(e));
        }
    }
}

// -k T'' = Q, T(0) = T0, k T'(L) = q: Neumann flux on the top face (apply_neumann_bcs)
void flux_profile() {
    const double lz = 600, k = 3.0, Q = 1e-6, T0 = 1280, q = 0.02;
    Mesh mesh = ImprovedMeshGenerator::generate_cube(4, 4, 4, 1000, 1000, lz);
    DofManager dofs(mesh.num_nodes(), 1);
    for (size_t i = 0; i < mesh.num_nodes(); ++i)
        if (std::fabs(mesh.nodes[i][2]) < 1.0) dofs.set_dirichlet_node(i, T0);
    CsMat K = Assembler::assemble_thermal_stiffness_parallel(mesh, dofs, k);
    std::vector<double> f = Assembler::assemble_thermal_load(mesh, dofs, Q);
    BoundaryConditions bcs;
    for (const BoundaryFace& face :
         Assembler::find_boundary_faces(mesh, [&](const Point3& p) { return std::fabs(p[2] - lz) < 1.0; }))
        bcs.add_neumann(face, q);
    Assembler::apply_neumann_bcs(mesh, f, bcs);
    auto kb = Assembler::apply_dirichlet_bcs(K, f, dofs);
    auto sol = ConjugateGradient().with_max_iterations(2000).with_tolerance(1e-12).solve(kb.first, kb.second);
    double err = 0, scale = 0;
    for (size_t i = 0; i < mesh.num_nodes(); ++i) {
        const double z = mesh.nodes[i][2];
        const double exact = T0 + (Q * lz + q) * z / k - Q * z * z / (2 * k);
        err = std::fmax(err, std::fabs(sol.first[i] - exact));
        scale = std::fmax(scale, std::fabs(exact));
    }
    expect(sol.second.converged && bcs.num_neumann_bcs() == 32 && err <= 1e-6 * scale,
           "Neumann flux profile 4^3: max error " + sci(err) + " (" + std::to_string(bcs.num_neumann_bcs()) +
               " top faces)");
}

// maxwell_stress_relaxation.rs: held uniaxial stress, deviatoric part decays by 1/(1 + dt/tau) per step
void maxwell_relaxation() {
    const double E = 100e9, nu = 0.25, eps0 = 1e-3;
    const MaxwellViscoelasticity m = MaxwellViscoelasticity::new_(E, nu, 1e19);
    const double dt = 0.5 * m.relaxation_time();
    Mesh mesh = ImprovedMeshGenerator::generate_cube(2, 2, 2, 1.0, 1.0, 1.0);
    DofManager dofs(mesh.num_nodes(), 3);
    for (size_t i = 0; i < mesh.num_nodes(); ++i) {
        const double x = mesh.nodes[i][0], y = mesh.nodes[i][1], z = mesh.nodes[i][2];
        const double dmin = std::fmin(std::fmin(std::fmin(x, 1 - x), std::fmin(y, 1 - y)), std::fmin(z, 1 - z));
        if (dmin < 1e-6) {
            dofs.set_dirichlet(dofs.global_dof(i, 0), -nu * eps0 * x);
            dofs.set_dirichlet(dofs.global_dof(i, 1), -nu * eps0 * y);
            dofs.set_dirichlet(dofs.global_dof(i, 2), eps0 * z);
        }
    }
    StressHistory sh(mesh.num_elements());
    const ConjugateGradient cg = ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-12);
    auto sys = Assembler::assemble_maxwell_viscoelastic_parallel(mesh, dofs, m, 1e-20, sh);
    auto kb = Assembler::apply_dirichlet_bcs(sys.first, std::vector<double>(dofs.total_dofs(), 0.0), dofs);
    std::vector<double> u = cg.solve(kb.first, kb.second).first;
    sh.stress = update_stresses_maxwell(mesh, m, std::vector<double>(u.size(), 0.0), u, 1e-20, sh);
    double worst = 0;
    for (int k = 1; k <= 3; ++k) {
        auto step = Assembler::assemble_maxwell_viscoelastic_parallel(mesh, dofs, m, dt, sh);
        auto sb = Assembler::apply_dirichlet_bcs(step.first, step.second, dofs);
        std::vector<double> un = cg.solve(sb.first, sb.second).first;
        sh.stress = update_stresses_maxwell(mesh, m, u, un, dt, sh);
        u = un;
        const double p = E * eps0 / 3, expect = p + 2 * p * std::pow(1.0 + dt / m.relaxation_time(), -k);
        for (const Voigt& s : sh.stress) worst = std::fmax(worst, std::fabs(s[2] - expect) / expect);
    }
    expect(worst < 1e-6, "Maxwell stress relaxation (3 backward-Euler steps): max rel error " + sci(worst));
}

void small_cg() {
    CsMat A = CsMat::from_arrays(2, 2, {0, 2, 4}, {0, 1, 0, 1}, {2.0, 1.0, 1.0, 2.0});
    auto s = ConjugateGradient().solve(A, {3.0, 3.0});
    expect(s.second.converged && std::fabs(s.first[0] - 1) < 1e-6 && std::fabs(s.first[1] - 1) < 1e-6,
           "2x2 CG converges to (1, 1)");
    CsMat D = CsMat::from_arrays(3, 3, {0, 1, 2, 3}, {0, 1, 2}, {2.0, 4.0, 8.0});
    auto d = ConjugateGradient().solve(D, {2.0, 4.0, 8.0});
    expect(d.second.converged && d.second.iterations == 0 && max_abs_diff(d.first, {1, 1, 1}) < 1e-14,
           "diagonal system: Jacobi solves it in 0 iterations");
    auto z = ConjugateGradient().solve(A, {0.0, 0.0});
    expect(z.second.converged && z.second.iterations == 0 && z.first[0] == 0 && z.first[1] == 0,
           "zero right-hand side returns zeros");
}

void patch_test() {
    const double L = 10e3, E = 100e9, nu = 0.25, s0 = 10e6;
    const double ezz = s0 / E, exx = -nu * s0 / E;
    Mesh mesh = ImprovedMeshGenerator::generate_cube(3, 3, 3, L, L, L);
    DofManager dofs(mesh.num_nodes(), 3);
    for (size_t i = 0; i < mesh.num_nodes(); ++i) {
        const double x = mesh.nodes[i][0], y = mesh.nodes[i][1], z = mesh.nodes[i][2];
        if (std::fabs(z) < 1.0 || std::fabs(z - L) < 1.0) dofs.set_dirichlet(dofs.global_dof(i, 2), ezz * z);
        if (std::fabs(x) < 1.0) dofs.set_dirichlet(dofs.global_dof(i, 0), exx * x);
        if (std::fabs(y) < 1.0) dofs.set_dirichlet(dofs.global_dof(i, 1), exx * y);
    }
    const IsotropicElasticity mat{E, nu};
    CsMat K = Assembler::assemble_elasticity_stiffness_parallel(mesh, dofs, mat);
    auto kb = Assembler::apply_dirichlet_bcs(K, std::vector<double>(dofs.total_dofs(), 0.0), dofs);
    auto sol = ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-12).solve(kb.first, kb.second);
    std::vector<double> exact(dofs.total_dofs());
    for (size_t i = 0; i < mesh.num_nodes(); ++i) {
        exact[3 * i] = exx * mesh.nodes[i][0];
        exact[3 * i + 1] = exx * mesh.nodes[i][1];
        exact[3 * i + 2] = ezz * mesh.nodes[i][2];
    }
    double scale = 0;
    for (double v : exact) scale = std::fmax(scale, std::fabs(v));
    expect(sol.second.converged && max_abs_diff(sol.first, exact) <= 1e-6 * scale, "elasticity patch test (CSR)");
    ElasticityOperator op(mesh, dofs, mat);
    auto mf = op.forward(std::vector<double>(dofs.total_dofs(), 0.0),
                         ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-12).with_precision(
                             Precision::Mixed));
    expect(mf.second.converged && max_abs_diff(mf.first, exact) <= 1e-6 * scale,
           "elasticity patch test (matrix-free, mixed precision)");
}

void errors() {
    Mesh line;
    for (int i = 0; i < 10; ++i) line.nodes.push_back({double(i), 0.0, 0.0});
    line.elements.push_back({0, 1, 2, 3, 4, 5, 6, 7, 8, 9});
    DofManager d1(10, 1);
    int code = GEO_OK;
    try {
        Assembler::assemble_thermal_stiffness_parallel(line, d1, 1.0);
    } catch (const Error& e) {
        code = e.code();
    }
    expect(code == GEO_ERR_SINGULAR_JACOBIAN, "singular Jacobian raises GEO_ERR_SINGULAR_JACOBIAN");
    Mesh cube = ImprovedMeshGenerator::generate_cube(1, 1, 1, 1.0, 1.0, 1.0);
    code = GEO_OK;
    try {
        DofManager d(cube.num_nodes(), 1);
        Assembler::assemble_elasticity_stiffness_parallel(cube, d, IsotropicElasticity{1e9, 0.2});
    } catch (const Error& e) {
        code = e.code();
    }
    expect(code == GEO_ERR_INVALID_ARG, "elasticity with 1 DOF per node raises GEO_ERR_INVALID_ARG");
    // non-convergence is reported, not thrown
    Mesh mesh = ImprovedMeshGenerator::generate_cube(4, 4, 4, 1000, 1000, 600);
    DofManager dofs = thermal_dofs(mesh, 600, 1280, 0);
    auto kb = Assembler::apply_dirichlet_bcs(Assembler::assemble_thermal_stiffness_parallel(mesh, dofs, 3.0),
                                             Assembler::assemble_thermal_load(mesh, dofs, 1e-6), dofs);
    auto s = ConjugateGradient().with_max_iterations(3).solve(kb.first, kb.second);
    expect(!s.second.converged && s.second.iterations == 3 && s.second.status == GEO_NOT_CONVERGED,
           "max_iterations reached: converged = false, no exception");
}

// The reference's 2x2 system (iterative.rs:491-504) through the CG siblings
void krylov_siblings() {
    const CsMat A = CsMat::from_arrays(2, 2, {0, 2, 4}, {0, 1, 0, 1}, {2.0, 1.0, 1.0, 2.0});
    const auto bi = BiCGSTAB().solve(A, {3.0, 3.0});
    const auto gm = GMRES().with_restart(5).solve(A, {3.0, 3.0});
    expect(bi.second.converged && std::fabs(bi.first[0] - 1.0) < 1e-6 && std::fabs(bi.first[1] - 1.0) < 1e-6,
           "BiCGSTAB on the 2x2 system");
    expect(gm.second.converged && std::fabs(gm.first[0] - 1.0) < 1e-6 && std::fabs(gm.first[1] - 1.0) < 1e-6,
           "GMRES on the 2x2 system");
    // direct.rs:103-122
    const auto lu = DirectSolver().solve(A, {3.0, 3.0});
    expect(lu.second.converged && lu.second.iterations == 0 && std::fabs(lu.first[0] - 1.0) < 1e-10 &&
               std::fabs(lu.first[1] - 1.0) < 1e-10,
           "DirectSolver on the 2x2 system");
    const CsMat S = CsMat::from_arrays(2, 2, {0, 2, 4}, {0, 1, 0, 1}, {1.0, 2.0, 2.0, 4.0});
    bool singular = false;
    try {
        DirectSolver().solve(S, {1.0, 1.0});
    } catch (const Error& e) {
        singular = e.code() == GEO_ERR_SINGULAR_MATRIX;
    }
    expect(singular, "DirectSolver raises GEO_ERR_SINGULAR_MATRIX on a singular matrix");
}

void adjoint_fd() {
    const double lz = 600;
    Mesh mesh = ImprovedMeshGenerator::generate_cube(4, 4, 3, 1000, 1000, lz);
    DofManager dofs = thermal_dofs(mesh, lz, 1280, 0);
    std::vector<double> lnk(mesh.num_elements());
    for (size_t e = 0; e < lnk.size(); ++e) lnk[e] = std::log(3.0) + 0.3 * std::sin(0.7 * double(e));
    auto expk = [](const std::vector<double>& v) {
        std::vector<double> k(v.size());
        for (size_t i = 0; i < v.size(); ++i) k[i] = std::exp(v[i]);
        return k;
    };
    const std::vector<double> f = Assembler::assemble_thermal_load(mesh, dofs, 1e-6);
    ThermalOperator op(mesh, dofs, expk(lnk));
    const ConjugateGradient tight = ConjugateGradient().with_max_iterations(20000).with_tolerance(1e-13);
    auto u = op.forward(f, tight).first;
    // J = 1/2 sum over free nodes with index % 7 == 0 of (u - (u0 + 1))^2
    std::vector<double> target(u.size()), dJ(u.size(), 0.0);
    std::vector<size_t> obs;
    for (size_t i = 0; i < u.size(); i += 7)
        if (!dofs.is_dirichlet(i)) obs.push_back(i);
    for (size_t i : obs) {
        target[i] = u[i] + 1.0;
        dJ[i] = u[i] - target[i];
    }
    auto J = [&](const std::vector<double>& uu) {
        double s = 0;
        for (size_t i : obs) s += 0.5 * (uu[i] - target[i]) * (uu[i] - target[i]);
        return s;
    };
    auto grad = op.vjp(dJ, &u, nullptr, tight).first;
    auto grad_r = op.vjp(dJ, nullptr, &f, tight).first;
    double gmax = 0;
    for (double g : grad) gmax = std::fmax(gmax, std::fabs(g));
    expect(max_abs_diff(grad, grad_r) <= 1e-7 * gmax, "vjp with stored u == vjp recomputing u");
    bool ok = true;
    const double h = 1e-6;
    for (size_t e : {size_t(3), size_t(50), size_t(111)}) {
        std::vector<double> lp = lnk, lm = lnk;
        lp[e] += h;
        lm[e] -= h;
        op.set_coefficients(expk(lp));
        const double jp = J(op.forward(f, tight).first);
        op.set_coefficients(expk(lm));
        const double jm = J(op.forward(f, tight).first);
        const double fd = (jp - jm) / (2 * h);
        ok = ok && std::fabs(grad[e] - fd) <= 1e-5 * std::fmax(std::fabs(fd), 1e-3 * gmax);
    }
    op.set_coefficients(expk(lnk));
    expect(ok, "adjoint dJ/d(ln k_e) agrees with central finite differences to 1e-5");
}

void device_mesh() {
    Context& ctx = Context::default_context();
    const Mesh hm = ImprovedMeshGenerator::generate_cube(5, 4, 3, 1000, 800, 600);
    Mesh dm = ImprovedMeshGenerator::generate_cube_device(ctx, 5, 4, 3, 1000, 800, 600);
    expect(!dm.host_resident() && dm.num_nodes() == hm.num_nodes() && dm.num_elements() == hm.num_elements(),
           "device mesh: sizes without a host copy");
    DofManager dofs(hm.num_nodes(), 1);
    const CsMat Kh = Assembler::assemble_thermal_stiffness_parallel(hm, dofs, 2.0);
    const CsMat Kd = Assembler::assemble_thermal_stiffness_parallel(dm, dofs, 2.0);
    std::vector<int64_t> ph, pd;
    std::vector<int32_t> ih, id;
    std::vector<double> vh, vd;
    Kh.to_host(ph, ih, vh);
    Kd.to_host(pd, id, vd);
    expect(ph == pd && ih == id && vh == vd, "device mesh assembles the same CSR as the host mesh");
    dm.download(ctx);
    bool same = dm.elements == hm.elements && dm.nodes.size() == hm.nodes.size();
    for (size_t i = 0; same && i < hm.nodes.size(); ++i)
        same = std::memcmp(dm.nodes[i].data(), hm.nodes[i].data(), sizeof(Point3)) == 0;
    expect(same, "device mesh downloads bit-identical to the host generator");
}

void vtu_output() {
    Mesh mesh = ImprovedMeshGenerator::generate_cube(2, 1, 1, 1000, 800, 600);
    std::vector<double> t(mesh.num_nodes(), 1.0);
    t[0] = 0.1 + 0.2;
    t[1] = -0.0;
    t[2] = 1e21;
    mesh.field_data.add_field({"T", t});
    mesh.cell_data.add_vector_field(VectorField::from_dof_vector("q", std::vector<double>(3 * mesh.num_elements(), 2.5e-7)));
    const std::string text = VtkWriter::render_vtu(mesh);
    expect(text.find("    <Piece NumberOfPoints=\"45\" NumberOfCells=\"12\">\n") != std::string::npos &&
               text.find("          0 0 0\n          500 0 0\n          1000 0 0\n") != std::string::npos,
           "VTU header and points as Rust prints them");
    expect(text.find("          0.30000000000000004 -0 1000000000000000000000 1 ") != std::string::npos &&
               text.find("0.00000025 0.00000025 0.00000025 ") != std::string::npos,
           "VTU field values printed as Rust's Display");
    const char* path = "host_api_test_out.vtu";
    const size_t n = VtkWriter::write_vtu(mesh, path);
    std::string back;
    if (FILE* fp = std::fopen(path, "rb")) {
        char buf[4096];
        size_t k;
        while ((k = std::fread(buf, 1, sizeof buf, fp)) > 0) back.append(buf, k);
        std::fclose(fp);
    }
    std::remove(path);
    expect(n == text.size() && back == text, "write_vtu streams the same bytes as render_vtu");
    const std::string legacy = VtkWriter::render(mesh, GEO_VTK_LEGACY);
    expect(legacy.rfind("# vtk DataFile Version 3.0\nTet10 Mesh generated by geo_simulator\nASCII\n", 0) == 0 &&
               legacy.find("\nCELLS 12 132\n10 ") != std::string::npos &&
               legacy.find("SCALARS T double 1\nLOOKUP_TABLE default\n0.30000000000000004\n-0\n") != std::string::npos,
           "legacy VTK layout as VtkWriter::write");
    const std::string nodal = VtkWriter::render(mesh, GEO_VTK_XML_NODAL);
    expect(nodal.find("Name=\"SoftenedCohesion\" format=\"ascii\">\n          0 0 ") != std::string::npos &&
               nodal.find("<CellData>") == std::string::npos,
           "nodal VTU: the named plasticity fields default to zero, no CellData");
}

}  // namespace

int main() {
    int n = 0;
    if (geo_device_count(&n) != GEO_OK || n < 1) {
        std::printf("no CUDA device\n");
        return 2;
    }
    try {
        small_cg();
        thermal_profile();
        patch_test();
        flux_profile();
        maxwell_relaxation();
        errors();
        adjoint_fd();
        krylov_siblings();
        device_mesh();
        vtu_output();
    } catch (const Error& e) {
        std::printf("FAIL unexpected geofem::Error %d: %s\n", e.code(), e.what());
        return 1;
    }
    std::printf("%s: %d failure(s)\n", g_failures ? "FAILED" : "PASSED", g_failures);
    return g_failures ? 1 : 0;
}
