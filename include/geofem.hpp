// geofem.hpp -- C++17 host API over the geo_fem.h C ABI, shaped like the Rust
// API of msahamed/geo_simulator's FEM hot path so that code written against
// the reference reads the same:
//
//   reference (Rust)                                   here (C++)
//   ImprovedMeshGenerator::generate_cube(..)           geofem::ImprovedMeshGenerator::generate_cube(..)
//     (src/mesh/mesh_generator_improved.rs:19-169)        and generate_cube_device(ctx, ..) (on the GPU)
//   DofManager::new(n, dpn), set_dirichlet(_node)      geofem::DofManager(n, dpn), set_dirichlet(_node)
//     (src/fem/dof.rs:37-140)
//   Assembler::assemble_thermal_stiffness_parallel     geofem::Assembler::assemble_thermal_stiffness_parallel
//     / assemble_thermal_load / apply_dirichlet_bcs      / assemble_thermal_load / apply_dirichlet_bcs
//     / assemble_elasticity_stiffness_parallel          / assemble_elasticity_stiffness_parallel
//     / assemble_gravity_load (src/fem/assembly.rs)      / assemble_gravity_load
//   IsotropicElasticity::new(E, nu)                    geofem::IsotropicElasticity{E, nu}
//   ConjugateGradient::new().with_*(..), Solver::solve geofem::ConjugateGradient().with_*(..).solve(A, b)
//     (src/linalg/iterative.rs:7-147)
//   BiCGSTAB / GMRES (src/linalg/iterative.rs:150-479) geofem::BiCGSTAB / GMRES
//   SolverStats (src/linalg/solver.rs:5-32)            geofem::SolverStats
//   CsMat<f64> (sprs)                                  geofem::CsMat (device-resident CSR)
//   FieldData / ScalarField / VectorField (mesh/fields.rs) geofem::FieldData / ScalarField / VectorField
//   VtkWriter::write / write_vtu / write_nodal_vtu     geofem::VtkWriter::write / write_vtu / write_nodal_vtu
//     (mesh/vtk_writer.rs:13-789)                        / render (GPU text)
//
// plus the matrix-free operators, the mixed-precision solve and the adjoint
// (geofem::ThermalOperator / ElasticityOperator with forward and vjp), which
// have no reference counterpart.
//
// Error behaviour: where the reference panics (singular Jacobian, wrong DOFs per
// node, bad arguments) these functions throw geofem::Error carrying the C status
// code and message. Non-convergence does not throw: as in the reference it is
// reported through SolverStats::converged (and SolverStats::status).
//
// Vectors are std::vector<double> in host memory; every call copies in and out
// and synchronises before returning. Meshes and DOF managers are uploaded to
// the GPU on first use and cached; call invalidate() after editing them.
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "geo_fem.h"

namespace geofem {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

class Context {
public:
    explicit Context(int device = 0) {
        geo_ctx* h = nullptr;
        const int rc = geo_ctx_create(device, &h);
        if (rc != GEO_OK) throw Error(rc, std::string("geo_ctx_create: ") + geo_last_error(nullptr));
        h_.reset(h);
    }
    // One context per device and host thread, created on first use.
    static Context& default_context(int device = 0) {
        thread_local std::vector<std::unique_ptr<Context>> ctxs;
        if ((int)ctxs.size() <= device) ctxs.resize(device + 1);
        if (!ctxs[device]) ctxs[device].reset(new Context(device));
        return *ctxs[device];
    }
    geo_ctx* get() const { return h_.get(); }
    // Throws unless rc is GEO_OK or one of the allowed codes; returns rc.
    int check(int rc, std::initializer_list<int> allow = {}) const {
        if (rc == GEO_OK) return rc;
        for (int a : allow)
            if (rc == a) return rc;
        throw Error(rc, geo_last_error(h_.get()));
    }

private:
    struct Del {
        void operator()(geo_ctx* c) const { geo_ctx_destroy(c); }
    };
    std::unique_ptr<geo_ctx, Del> h_;
};

// ---------------------------------------------------------------- mesh and DOFs
using Point3 = std::array<double, 3>;
using Tet10 = std::array<int32_t, 10>;  // [v0 v1 v2 v3 e01 e12 e20 e03 e13 e23]

// mesh/fields.rs:4-137. The reference keys HashMaps (iteration order unspecified);
// these keep insertion order, which VtkWriter writes.
struct ScalarField {
    std::string name;
    std::vector<double> data;
};
struct VectorField {
    std::string name;
    std::vector<Point3> data;
    // fields.rs:54-66: interleaved [x0 y0 z0 x1 ...]
    static VectorField from_dof_vector(const std::string& name, const std::vector<double>& dofs) {
        if (dofs.size() % 3) throw std::invalid_argument("DOF vector must have 3*n entries for vector field");
        VectorField f{name, std::vector<Point3>(dofs.size() / 3)};
        for (size_t i = 0; i < f.data.size(); ++i) f.data[i] = {dofs[3 * i], dofs[3 * i + 1], dofs[3 * i + 2]};
        return f;
    }
};
struct FieldData {
    std::vector<ScalarField> scalar_fields;
    std::vector<VectorField> vector_fields;
    void add_field(ScalarField f) { put(scalar_fields, std::move(f)); }
    void add_vector_field(VectorField f) { put(vector_fields, std::move(f)); }
    bool is_empty() const { return scalar_fields.empty() && vector_fields.empty(); }

private:
    template <class F>
    static void put(std::vector<F>& v, F f) {  // HashMap::insert: a field of the same name is replaced
        for (auto& g : v)
            if (g.name == f.name) {
                g = std::move(f);
                return;
            }
        v.push_back(std::move(f));
    }
};

class Mesh {
public:
    std::vector<Point3> nodes;     // geometry.nodes
    std::vector<Tet10> elements;   // connectivity.tet10_elements
    FieldData field_data;          // point data written by VtkWriter
    FieldData cell_data;           // cell data written by VtkWriter

    Mesh() = default;
    Mesh(std::vector<Point3> n, std::vector<Tet10> e) : nodes(std::move(n)), elements(std::move(e)) {}
    // A mesh that exists only on the device (ImprovedMeshGenerator::generate_cube_device):
    // nodes/elements stay empty until download() copies them out.
    static Mesh from_device(Context& ctx, geo_mesh* m) {
        Mesh out;
        out.dev_.reset(m, [](geo_mesh* p) { geo_mesh_destroy(p); });
        out.dev_ctx_ = ctx.get();
        int64_t nn = 0, ne = 0;
        ctx.check(geo_mesh_size(m, &nn, &ne));
        out.dev_nodes_ = (size_t)nn;
        out.dev_elems_ = (size_t)ne;
        return out;
    }
    size_t num_nodes() const { return nodes.empty() && dev_ ? dev_nodes_ : nodes.size(); }
    size_t num_elements() const { return elements.empty() && dev_ ? dev_elems_ : elements.size(); }
    bool host_resident() const { return !nodes.empty() || !dev_; }
    // Fills nodes/elements from the device copy (no-op for a host mesh).
    void download(Context& ctx) {
        if (host_resident()) return;
        nodes.resize(dev_nodes_);
        elements.resize(dev_elems_);
        ctx.check(geo_mesh_download(dev_.get(), nodes[0].data(), elements[0].data()));
    }
    void invalidate() {
        if (host_resident()) dev_.reset();
    }

    const geo_mesh* handle(Context& ctx) const {
        if (dev_ && !host_resident() && dev_ctx_ != ctx.get())
            throw Error(GEO_ERR_INVALID_ARG, "device-only mesh used with another context: download() it first");
        if (!dev_ || dev_ctx_ != ctx.get()) {
            geo_mesh* m = nullptr;
            ctx.check(geo_mesh_create(ctx.get(), (int64_t)nodes.size(), nodes.empty() ? nullptr : nodes[0].data(),
                                      (int64_t)elements.size(), elements.empty() ? nullptr : elements[0].data(),
                                      &m));
            dev_.reset(m, [](geo_mesh* p) { geo_mesh_destroy(p); });
            dev_ctx_ = ctx.get();
        }
        return dev_.get();
    }

private:
    mutable std::shared_ptr<geo_mesh> dev_;
    mutable const geo_ctx* dev_ctx_ = nullptr;
    size_t dev_nodes_ = 0, dev_elems_ = 0;
};

struct ImprovedMeshGenerator {
    // mesh_generator_improved.rs:19-169: (2nx+1)(2ny+1)(2nz+1) nodes, 6 nx ny nz Tet10
    static Mesh generate_cube(int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz) {
        int64_t nn = 0, ne = 0;
        int rc = geo_generate_cube_size(nx, ny, nz, &nn, &ne);
        if (rc != GEO_OK) throw Error(rc, "generate_cube: invalid size");
        Mesh m;
        m.nodes.resize((size_t)nn);
        m.elements.resize((size_t)ne);
        rc = geo_generate_cube(nx, ny, nz, lx, ly, lz, m.nodes[0].data(), m.elements[0].data());
        if (rc != GEO_OK) throw Error(rc, "generate_cube failed");
        return m;
    }
    // The same mesh built in device memory (geo_mesh_generate_cube); see Mesh::from_device.
    static Mesh generate_cube_device(Context& ctx, int64_t nx, int64_t ny, int64_t nz, double lx, double ly,
                                     double lz) {
        geo_mesh* m = nullptr;
        ctx.check(geo_mesh_generate_cube(ctx.get(), nx, ny, nz, lx, ly, lz, &m));
        return Mesh::from_device(ctx, m);
    }
};

// mesh/vtk_writer.rs:13-789: the VTK writers, with the text rendered on the GPU byte for byte.
struct VtkWriter {
    // VtkWriter::write (vtk_writer.rs:13-101): legacy ASCII .vtk
    static size_t write(const Mesh& mesh, const std::string& filename, Context& ctx = Context::default_context()) {
        return to_file(mesh, GEO_VTK_LEGACY, filename, ctx);
    }
    // VtkWriter::write_vtu (vtk_writer.rs:104-265)
    static size_t write_vtu(const Mesh& mesh, const std::string& filename,
                            Context& ctx = Context::default_context()) {
        return to_file(mesh, GEO_VTK_XML, filename, ctx);
    }
    // VtkWriter::write_nodal_vtu (vtk_writer.rs:531-789); the reference ignores its tracers
    static size_t write_nodal_vtu(const Mesh& mesh, const std::string& filename,
                                  Context& ctx = Context::default_context()) {
        return to_file(mesh, GEO_VTK_XML_NODAL, filename, ctx);
    }
    // the text of one of the writers (GEO_VTK_LEGACY / GEO_VTK_XML / GEO_VTK_XML_NODAL) in memory
    static std::string render(const Mesh& mesh, int format = GEO_VTK_XML, Context& ctx = Context::default_context()) {
        Fields f(mesh);
        int64_t size = 0;
        ctx.check(geo_vtk_render(ctx.get(), mesh.handle(ctx), format, f.point.data(), (int32_t)f.point.size(),
                                 f.cell.data(), (int32_t)f.cell.size(), nullptr, 0, &size));
        std::string out((size_t)size, '\0');
        ctx.check(geo_vtk_render(ctx.get(), mesh.handle(ctx), format, f.point.data(), (int32_t)f.point.size(),
                                 f.cell.data(), (int32_t)f.cell.size(), &out[0], size, &size));
        return out;
    }
    static std::string render_vtu(const Mesh& mesh, Context& ctx = Context::default_context()) {
        return render(mesh, GEO_VTK_XML, ctx);
    }

private:
    static size_t to_file(const Mesh& mesh, int format, const std::string& filename, Context& ctx) {
        Fields f(mesh);
        int64_t size = 0;
        ctx.check(geo_write_vtk(ctx.get(), mesh.handle(ctx), format, f.point.data(), (int32_t)f.point.size(),
                                f.cell.data(), (int32_t)f.cell.size(), filename.c_str(), &size));
        return (size_t)size;
    }
    struct Fields {
        std::vector<geo_vtu_field> point, cell;
        explicit Fields(const Mesh& m) {
            add(point, m.field_data);
            add(cell, m.cell_data);
        }
        static void add(std::vector<geo_vtu_field>& v, const FieldData& fd) {
            for (const auto& f : fd.scalar_fields) v.push_back({f.name.c_str(), f.data.data(), (int64_t)f.data.size(), 1});
            for (const auto& f : fd.vector_fields)
                v.push_back({f.name.c_str(), f.data.empty() ? nullptr : f.data[0].data(), (int64_t)f.data.size(), 3});
        }
    };
};

class DofManager {
public:
    DofManager(size_t num_nodes, int dofs_per_node)
        : n_nodes_(num_nodes), dpn_(dofs_per_node), mask_(num_nodes * dofs_per_node, 0),
          vals_(num_nodes * dofs_per_node, 0.0) {}
    size_t global_dof(size_t node_id, int local_dof) const {
        if (local_dof < 0 || local_dof >= dpn_) throw Error(GEO_ERR_INVALID_ARG, "local DOF out of range");
        return node_id * dpn_ + local_dof;
    }
    void set_dirichlet(size_t dof, double value) {
        if (dof >= mask_.size()) throw Error(GEO_ERR_INVALID_ARG, "DOF out of range");
        mask_[dof] = 1;
        vals_[dof] = value;
        dev_.reset();
    }
    // every DOF of the node (dof.rs:125-130)
    void set_dirichlet_node(size_t node_id, double value) {
        for (int c = 0; c < dpn_; ++c) set_dirichlet(global_dof(node_id, c), value);
    }
    bool is_dirichlet(size_t dof) const { return dof < mask_.size() && mask_[dof] != 0; }
    double get_dirichlet_value(size_t dof) const { return is_dirichlet(dof) ? vals_[dof] : 0.0; }
    size_t total_dofs() const { return mask_.size(); }
    size_t num_constrained_dofs() const {
        size_t c = 0;
        for (uint8_t m : mask_) c += m != 0;
        return c;
    }
    size_t num_free_dofs() const { return total_dofs() - num_constrained_dofs(); }
    int dofs_per_node() const { return dpn_; }
    size_t num_nodes() const { return n_nodes_; }

    const geo_dofs* handle(Context& ctx) const {
        if (!dev_ || dev_ctx_ != ctx.get()) {
            geo_dofs* d = nullptr;
            ctx.check(geo_dofs_create(ctx.get(), (int64_t)n_nodes_, dpn_, mask_.data(), vals_.data(), &d));
            dev_.reset(d, [](geo_dofs* p) { geo_dofs_destroy(p); });
            dev_ctx_ = ctx.get();
        }
        return dev_.get();
    }

private:
    size_t n_nodes_;
    int dpn_;
    std::vector<uint8_t> mask_;
    std::vector<double> vals_;
    mutable std::shared_ptr<geo_dofs> dev_;
    mutable const geo_ctx* dev_ctx_ = nullptr;
};

struct IsotropicElasticity {
    double youngs_modulus;
    double poisson_ratio;
    static IsotropicElasticity new_(double E, double nu) { return {E, nu}; }
};

// mechanics/constitutive.rs:286-395
struct MaxwellViscoelasticity {
    double youngs_modulus;
    double poisson_ratio;
    double viscosity;
    static MaxwellViscoelasticity new_(double E, double nu, double mu) {
        if (!(E > 0) || !(nu > -1.0 && nu < 0.5) || !(mu > 0))
            throw Error(GEO_ERR_INVALID_ARG, "invalid Maxwell material parameters");
        return {E, nu, mu};
    }
    double shear_modulus() const { return youngs_modulus / (2.0 * (1.0 + poisson_ratio)); }
    double relaxation_time() const { return viscosity / shear_modulus(); }
};

// mesh/state.rs:12-75: Voigt stress [xx yy zz xy yz zx] per element
using Voigt = std::array<double, 6>;
struct StressHistory {
    std::vector<Voigt> stress;
    explicit StressHistory(size_t n_elements = 0) : stress(n_elements, Voigt{0, 0, 0, 0, 0, 0}) {}
};

// ---------------------------------------------------------------- CSR
class CsMat {
public:
    CsMat() = default;
    CsMat(geo_csr* h, Context* ctx) : h_(h, [](geo_csr* p) { geo_csr_destroy(p); }), ctx_(ctx) {}
    // from host CSR arrays (sorted column indices per row)
    static CsMat from_arrays(int64_t rows, int64_t cols, const std::vector<int64_t>& indptr,
                             const std::vector<int32_t>& indices, const std::vector<double>& data,
                             Context& ctx = Context::default_context()) {
        geo_csr* h = nullptr;
        ctx.check(geo_csr_create(ctx.get(), rows, cols, (int64_t)data.size(), indptr.data(), indices.data(),
                                 data.data(), &h));
        return CsMat(h, &ctx);
    }
    int64_t rows() const { return info()[0]; }
    int64_t cols() const { return info()[1]; }
    int64_t nnz() const { return info()[2]; }
    void to_host(std::vector<int64_t>& indptr, std::vector<int32_t>& indices, std::vector<double>& data) const {
        const auto i = info();
        indptr.resize((size_t)i[0] + 1);
        indices.resize((size_t)i[2]);
        data.resize((size_t)i[2]);
        ctx_->check(geo_csr_copy(h_.get(), indptr.data(), indices.data(), data.data()));
    }
    // LinearOperator::apply (solver.rs:61-73)
    std::vector<double> apply(const std::vector<double>& x) const {
        std::vector<double> y((size_t)rows());
        ctx_->check(geo_csr_apply(ctx_->get(), h_.get(), x.data(), y.data()));
        return y;
    }
    const geo_csr* get() const { return h_.get(); }
    Context* context() const { return ctx_; }

private:
    std::array<int64_t, 3> info() const {
        std::array<int64_t, 3> v{0, 0, 0};
        ctx_->check(geo_csr_info(h_.get(), &v[0], &v[1], &v[2]));
        return v;
    }
    std::shared_ptr<geo_csr> h_;
    Context* ctx_ = nullptr;
};

// ---------------------------------------------------------------- Neumann boundary
// boundary.rs:9-59: a face is (element, local face), local face f opposite vertex f
struct BoundaryFace {
    int32_t element_id;
    int32_t local_face_id;
};

class BoundaryConditions {
public:
    void add_neumann(BoundaryFace face, double flux) {
        faces_.push_back(face);
        flux_.push_back(flux);
    }
    size_t num_neumann_bcs() const { return faces_.size(); }
    const std::vector<BoundaryFace>& faces() const { return faces_; }
    const std::vector<double>& fluxes() const { return flux_; }

private:
    std::vector<BoundaryFace> faces_;
    std::vector<double> flux_;
};

struct Tet10Face {
    std::array<int32_t, 6> nodes;  // 3 vertices then 3 edge midpoints (boundary.rs:89-130)
    static Tet10Face from_element_face(const Tet10& element_nodes, int local_face) {
        static const int kFace[4][6] = {{1, 2, 3, 5, 9, 8}, {0, 2, 3, 6, 9, 7}, {0, 1, 3, 4, 8, 7}, {0, 1, 2, 4, 5, 6}};
        if (local_face < 0 || local_face > 3) throw Error(GEO_ERR_INVALID_ARG, "Invalid face index for tet10");
        Tet10Face f;
        for (int i = 0; i < 6; ++i) f.nodes[i] = element_nodes[kFace[local_face][i]];
        return f;
    }
};

// ---------------------------------------------------------------- assembly
struct Assembler {
    // assembly.rs:287-309: faces whose 6 nodes all satisfy the condition, in (element, face) order
    static std::vector<BoundaryFace> find_boundary_faces(const Mesh& mesh,
                                                         const std::function<bool(const Point3&)>& condition,
                                                         Context& ctx = Context::default_context()) {
        if (!mesh.host_resident())
            throw Error(GEO_ERR_INVALID_ARG, "find_boundary_faces needs node coordinates: download() the mesh first");
        std::vector<uint8_t> mask(mesh.num_nodes());
        for (size_t i = 0; i < mask.size(); ++i) mask[i] = condition(mesh.nodes[i]) ? 1 : 0;
        int64_t n = 0;
        ctx.check(geo_find_boundary_faces(ctx.get(), mesh.handle(ctx), mask.data(), 0, nullptr, &n));
        std::vector<BoundaryFace> faces((size_t)n);
        if (n)
            ctx.check(geo_find_boundary_faces(ctx.get(), mesh.handle(ctx), mask.data(), n,
                                              reinterpret_cast<int32_t*>(faces.data()), &n));
        return faces;
    }
    // assembly.rs:248-274: f[node] += face flux contributions
    static void apply_neumann_bcs(const Mesh& mesh, std::vector<double>& f, const BoundaryConditions& bcs,
                                  Context& ctx = Context::default_context()) {
        if (f.size() < mesh.num_nodes()) throw Error(GEO_ERR_INVALID_ARG, "f shorter than the node count");
        ctx.check(geo_apply_neumann_bcs(ctx.get(), mesh.handle(ctx), (int64_t)bcs.num_neumann_bcs(),
                                        reinterpret_cast<const int32_t*>(bcs.faces().data()), bcs.fluxes().data(),
                                        0.0, (int64_t)f.size(), f.data()));
    }
    // assembly.rs:69-117 (uniform conductivity) and the per-element variant
    static CsMat assemble_thermal_stiffness_parallel(const Mesh& mesh, const DofManager& dofs, double conductivity,
                                                     Context& ctx = Context::default_context()) {
        return thermal_k(mesh, dofs, nullptr, conductivity, ctx);
    }
    static CsMat assemble_thermal_stiffness_parallel(const Mesh& mesh, const DofManager& dofs,
                                                     const std::vector<double>& k_e,
                                                     Context& ctx = Context::default_context()) {
        size_check(k_e.size(), mesh.num_elements(), "k_e");
        return thermal_k(mesh, dofs, k_e.data(), 0.0, ctx);
    }
    // assembly.rs:130-154
    static std::vector<double> assemble_thermal_load(const Mesh& mesh, const DofManager& dofs, double source,
                                                     Context& ctx = Context::default_context()) {
        std::vector<double> f(dofs.total_dofs());
        ctx.check(geo_assemble_thermal_load(ctx.get(), mesh.handle(ctx), dofs.handle(ctx), source, f.data()));
        return f;
    }
    // assembly.rs:168-230
    static std::pair<CsMat, std::vector<double>> apply_dirichlet_bcs(const CsMat& K, const std::vector<double>& f,
                                                                     const DofManager& dofs) {
        Context& ctx = *K.context();
        size_check(f.size(), dofs.total_dofs(), "f");
        geo_csr* kb = nullptr;
        std::vector<double> fb(f.size());
        ctx.check(geo_apply_dirichlet_bcs(ctx.get(), K.get(), f.data(), dofs.handle(ctx), &kb, fb.data()));
        return {CsMat(kb, &ctx), std::move(fb)};
    }
    // assembly.rs:389-437 (throws unless 3 DOFs per node, as the reference asserts)
    static CsMat assemble_elasticity_stiffness_parallel(const Mesh& mesh, const DofManager& dofs,
                                                        const IsotropicElasticity& mat,
                                                        const std::vector<double>* E_e = nullptr,
                                                        Context& ctx = Context::default_context()) {
        if (E_e) size_check(E_e->size(), mesh.num_elements(), "E_e");
        geo_csr* k = nullptr;
        ctx.check(geo_assemble_elasticity_stiffness(ctx.get(), mesh.handle(ctx), dofs.handle(ctx),
                                                    E_e ? E_e->data() : nullptr, mat.youngs_modulus,
                                                    mat.poisson_ratio, &k));
        return CsMat(k, &ctx);
    }
    // the history force of assemble_maxwell_viscoelastic_parallel (assembly.rs:959-1020)
    static std::vector<double> maxwell_history_force(const Mesh& mesh, const StressHistory& sh,
                                                     Context& ctx = Context::default_context()) {
        size_check(sh.stress.size(), mesh.num_elements(), "stress history");
        std::vector<double> f(3 * mesh.num_nodes());
        ctx.check(geo_maxwell_history_force(ctx.get(), mesh.handle(ctx), sh.stress[0].data(), f.data()));
        return f;
    }
    // assembly.rs:959-1020: (elastic K, f_history)
    static std::pair<CsMat, std::vector<double>> assemble_maxwell_viscoelastic_parallel(
        const Mesh& mesh, const DofManager& dofs, const MaxwellViscoelasticity& m, double dt, const StressHistory& sh,
        Context& ctx = Context::default_context()) {
        size_check(sh.stress.size(), mesh.num_elements(), "stress history");
        geo_csr* k = nullptr;
        std::vector<double> f(dofs.total_dofs());
        ctx.check(geo_assemble_maxwell_viscoelastic(ctx.get(), mesh.handle(ctx), dofs.handle(ctx), m.youngs_modulus,
                                                    m.poisson_ratio, m.viscosity, dt, sh.stress[0].data(), &k,
                                                    f.data()));
        return {CsMat(k, &ctx), std::move(f)};
    }
    // assembly.rs:906-937
    static std::vector<double> assemble_gravity_load(const Mesh& mesh, const DofManager& dofs, double density,
                                                     const std::array<double, 3>& gravity,
                                                     Context& ctx = Context::default_context()) {
        std::vector<double> f(dofs.total_dofs());
        ctx.check(geo_assemble_gravity_load(ctx.get(), mesh.handle(ctx), dofs.handle(ctx), density, gravity.data(),
                                            f.data()));
        return f;
    }

private:
    static CsMat thermal_k(const Mesh& mesh, const DofManager& dofs, const double* k_e, double k, Context& ctx) {
        geo_csr* h = nullptr;
        ctx.check(geo_assemble_thermal_stiffness(ctx.get(), mesh.handle(ctx), dofs.handle(ctx), k_e, k, &h));
        return CsMat(h, &ctx);
    }
    static void size_check(size_t got, size_t want, const char* what) {
        if (got != want) throw Error(GEO_ERR_INVALID_ARG, std::string(what) + " has the wrong length");
    }
};

// mechanics/stress_update.rs:39-143: stresses after the step u_n -> u_next
inline std::vector<Voigt> update_stresses_maxwell(const Mesh& mesh, const MaxwellViscoelasticity& m,
                                                  const std::vector<double>& u_n, const std::vector<double>& u_next,
                                                  double dt, const StressHistory& sh,
                                                  Context& ctx = Context::default_context()) {
    std::vector<Voigt> out(mesh.num_elements());
    ctx.check(geo_update_stresses_maxwell(ctx.get(), mesh.handle(ctx), m.youngs_modulus, m.poisson_ratio, m.viscosity,
                                          u_n.data(), u_next.data(), dt, sh.stress[0].data(), out[0].data()));
    return out;
}

// ---------------------------------------------------------------- solver
struct SolverStats {
    int64_t iterations = 0;
    double residual_norm = 0.0;
    double relative_residual = 0.0;
    bool converged = false;
    double solve_time = 0.0;
    // extensions
    int status = GEO_OK;
    int64_t fp64_residual_updates = 0;
    int64_t kernel_launches = 0;

    static SolverStats from_c(const geo_solver_stats& s) {
        SolverStats r;
        r.iterations = s.iterations;
        r.residual_norm = s.residual_norm;
        r.relative_residual = s.relative_residual;
        r.converged = s.converged != 0;
        r.solve_time = s.solve_time;
        r.status = s.status;
        r.fp64_residual_updates = s.fp64_residual_updates;
        r.kernel_launches = s.kernel_launches;
        return r;
    }
};

enum class Precision { FP64 = GEO_PRECISION_FP64, Mixed = GEO_PRECISION_MIXED };

class ConjugateGradient {
public:
    ConjugateGradient() { geo_cg_opts_default(&o_); }
    ConjugateGradient& with_max_iterations(int64_t n) { o_.max_iterations = n; return *this; }
    ConjugateGradient& with_tolerance(double t) { o_.tolerance = t; return *this; }
    ConjugateGradient& with_abs_tolerance(double t) { o_.abs_tolerance = t; return *this; }
    ConjugateGradient& with_preconditioner(bool on) { o_.use_preconditioner = on ? 1 : 0; return *this; }
    // matrix-free operators only: FP64 (the drop-in) or mixed FP32/FP64
    ConjugateGradient& with_precision(Precision p) { o_.precision = (int32_t)p; return *this; }
    const geo_cg_opts& opts() const { return o_; }

    // Solver::solve (iterative.rs:123-131): x0 = 0, Jacobi-PCG on the assembled CSR
    std::pair<std::vector<double>, SolverStats> solve(const CsMat& A, const std::vector<double>& b) const {
        Context& ctx = *A.context();
        if ((int64_t)b.size() != A.rows()) throw Error(GEO_ERR_INVALID_ARG, "b has the wrong length");
        std::vector<double> x(b.size());
        geo_solver_stats st{};
        ctx.check(geo_cg_solve(ctx.get(), A.get(), b.data(), &o_, x.data(), &st),
                  {GEO_NOT_CONVERGED, GEO_ERR_BREAKDOWN});
        return {std::move(x), SolverStats::from_c(st)};
    }

private:
    geo_cg_opts o_;
};

// BiCGSTAB (iterative.rs:150-301) and restarted GMRES (:303-479) on the assembled
// CSR, FP64, right-preconditioned with Jacobi or the identity
class BiCGSTAB {
public:
    BiCGSTAB() { geo_cg_opts_default(&o_); }
    BiCGSTAB& with_max_iterations(int64_t n) { o_.max_iterations = n; return *this; }
    BiCGSTAB& with_tolerance(double t) { o_.tolerance = t; return *this; }
    BiCGSTAB& with_abs_tolerance(double t) { o_.abs_tolerance = t; return *this; }
    BiCGSTAB& with_preconditioner(bool on) { o_.use_preconditioner = on ? 1 : 0; return *this; }
    std::pair<std::vector<double>, SolverStats> solve(const CsMat& A, const std::vector<double>& b) const {
        Context& ctx = *A.context();
        if ((int64_t)b.size() != A.rows()) throw Error(GEO_ERR_INVALID_ARG, "b has the wrong length");
        std::vector<double> x(b.size());
        geo_solver_stats st{};
        ctx.check(geo_bicgstab_solve(ctx.get(), A.get(), b.data(), &o_, x.data(), &st),
                  {GEO_NOT_CONVERGED, GEO_ERR_BREAKDOWN});
        return {std::move(x), SolverStats::from_c(st)};
    }

private:
    geo_cg_opts o_;
};

// DirectSolver (linalg/direct.rs:9-95): dense LU with partial pivoting on the
// device. A singular matrix throws Error(GEO_ERR_SINGULAR_MATRIX), where the
// reference panics; the tolerances are fixed at 0 as there.
class DirectSolver {
public:
    std::pair<std::vector<double>, SolverStats> solve(const CsMat& A, const std::vector<double>& b) const {
        Context& ctx = *A.context();
        if ((int64_t)b.size() != A.rows()) throw Error(GEO_ERR_INVALID_ARG, "b has the wrong length");
        std::vector<double> x(b.size());
        geo_solver_stats st{};
        ctx.check(geo_direct_solve(ctx.get(), A.get(), b.data(), x.data(), &st));
        return {std::move(x), SolverStats::from_c(st)};
    }
    const char* name() const { return "Direct (Sparse LU)"; }
    double tolerance() const { return 0.0; }
    double abs_tolerance() const { return 0.0; }
    void set_tolerance(double) {}
    void set_abs_tolerance(double) {}
};

class GMRES {
public:
    GMRES() { geo_cg_opts_default(&o_); }
    GMRES& with_restart(int m) { restart_ = m; return *this; }
    GMRES& with_max_iterations(int64_t n) { o_.max_iterations = n; return *this; }
    GMRES& with_tolerance(double t) { o_.tolerance = t; return *this; }
    GMRES& with_abs_tolerance(double t) { o_.abs_tolerance = t; return *this; }
    GMRES& with_preconditioner(bool on) { o_.use_preconditioner = on ? 1 : 0; return *this; }
    std::pair<std::vector<double>, SolverStats> solve(const CsMat& A, const std::vector<double>& b) const {
        Context& ctx = *A.context();
        if ((int64_t)b.size() != A.rows()) throw Error(GEO_ERR_INVALID_ARG, "b has the wrong length");
        std::vector<double> x(b.size());
        geo_solver_stats st{};
        ctx.check(geo_gmres_solve(ctx.get(), A.get(), b.data(), &o_, restart_, x.data(), &st),
                  {GEO_NOT_CONVERGED, GEO_ERR_BREAKDOWN});
        return {std::move(x), SolverStats::from_c(st)};
    }

private:
    geo_cg_opts o_;
    int restart_ = 10;  // the reference's default
};

// ---------------------------------------------------------------- matrix-free operators
// The Dirichlet-eliminated operator K_bc, applied without forming it; solve()
// replaces Solver::solve_with_operator (solver.rs:112-120), forward/vjp give the
// solution and the adjoint gradient dJ/d(ln coef_e).
class MatFreeOperator {
public:
    size_t rows() const {
        int64_t n = 0;
        geo_op_info(h_.get(), &n, nullptr, nullptr);
        return (size_t)n;
    }
    double char_diag() const {
        double cd = 0;
        geo_op_info(h_.get(), nullptr, nullptr, &cd);
        return cd;
    }
    void set_coefficients(const std::vector<double>& coef_e) {
        ctx_->check(geo_op_set_coefficients(h_.get(), coef_e.data(), 0.0));
    }
    std::vector<double> apply(const std::vector<double>& x, Precision p = Precision::FP64) const {
        std::vector<double> y(rows());
        ctx_->check(geo_op_apply(h_.get(), x.data(), y.data(), (int32_t)p));
        return y;
    }
    std::vector<double> lift_rhs(const std::vector<double>& f) const {
        std::vector<double> fb(rows());
        ctx_->check(geo_op_lift_rhs(h_.get(), f.data(), fb.data()));
        return fb;
    }
    std::vector<double> diagonal() const {
        std::vector<double> d(rows());
        ctx_->check(geo_op_diagonal(h_.get(), d.data()));
        return d;
    }
    // K_bc x = b_bc (b already Dirichlet-lifted)
    std::pair<std::vector<double>, SolverStats> solve(const std::vector<double>& b_bc,
                                                      const ConjugateGradient& cg = ConjugateGradient()) const {
        std::vector<double> x(rows());
        geo_solver_stats st{};
        ctx_->check(geo_cg_solve_matfree(h_.get(), b_bc.data(), &cg.opts(), x.data(), &st),
                    {GEO_NOT_CONVERGED, GEO_ERR_BREAKDOWN});
        return {std::move(x), SolverStats::from_c(st)};
    }
    // u = K_bc^{-1} lift(f)
    std::pair<std::vector<double>, SolverStats> forward(const std::vector<double>& f,
                                                        const ConjugateGradient& cg = ConjugateGradient()) const {
        std::vector<double> u(rows());
        geo_solver_stats st{};
        ctx_->check(geo_forward(h_.get(), f.data(), &cg.opts(), u.data(), &st), {GEO_NOT_CONVERGED, GEO_ERR_BREAKDOWN});
        return {std::move(u), SolverStats::from_c(st)};
    }
    // dJ/d(ln coef_e) given dJ/du; pass u = nullptr to recompute the forward solution from f
    std::pair<std::vector<double>, SolverStats> vjp(const std::vector<double>& dJ_du, const std::vector<double>* u,
                                                    const std::vector<double>* f,
                                                    const ConjugateGradient& cg = ConjugateGradient()) const {
        int64_t ne = 0;
        geo_op_info(h_.get(), nullptr, &ne, nullptr);
        std::vector<double> g((size_t)ne);
        geo_solver_stats st{};
        ctx_->check(geo_vjp(h_.get(), f ? f->data() : nullptr, u ? u->data() : nullptr, dJ_du.data(), &cg.opts(),
                            g.data(), &st),
                    {GEO_NOT_CONVERGED, GEO_ERR_BREAKDOWN});
        return {std::move(g), SolverStats::from_c(st)};
    }
    geo_op* get() const { return h_.get(); }

protected:
    MatFreeOperator(geo_op* h, Context* ctx) : h_(h, [](geo_op* p) { geo_op_destroy(p); }), ctx_(ctx) {}
    std::shared_ptr<geo_op> h_;
    Context* ctx_;
};

class ThermalOperator : public MatFreeOperator {
public:
    ThermalOperator(const Mesh& mesh, const DofManager& dofs, double conductivity,
                    Context& ctx = Context::default_context())
        : MatFreeOperator(create(mesh, dofs, nullptr, conductivity, ctx), &ctx) {}
    ThermalOperator(const Mesh& mesh, const DofManager& dofs, const std::vector<double>& k_e,
                    Context& ctx = Context::default_context())
        : MatFreeOperator(create(mesh, dofs, k_e.data(), 0.0, ctx), &ctx) {}

private:
    static geo_op* create(const Mesh& m, const DofManager& d, const double* k_e, double k, Context& ctx) {
        geo_op* h = nullptr;
        ctx.check(geo_thermal_operator_create(ctx.get(), m.handle(ctx), d.handle(ctx), k_e, k, &h));
        return h;
    }
};

class ElasticityOperator : public MatFreeOperator {
public:
    ElasticityOperator(const Mesh& mesh, const DofManager& dofs, const IsotropicElasticity& mat,
                       const std::vector<double>* E_e = nullptr, Context& ctx = Context::default_context())
        : MatFreeOperator(create(mesh, dofs, mat, E_e, ctx), &ctx) {}

private:
    static geo_op* create(const Mesh& m, const DofManager& d, const IsotropicElasticity& mat,
                          const std::vector<double>* E_e, Context& ctx) {
        geo_op* h = nullptr;
        ctx.check(geo_elasticity_operator_create(ctx.get(), m.handle(ctx), d.handle(ctx),
                                                 E_e ? E_e->data() : nullptr, mat.youngs_modulus,
                                                 mat.poisson_ratio, &h));
        return h;
    }
};

}  // namespace geofem
