/*
 * CPU oracle for the GeoSimulator Tet10 hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference's arithmetic (msahamed/geo_simulator,
 * Rust), used by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py as the checker. The product library (geo_simulator_b200/libgeofem.so)
 * never links, loads or calls it.
 *
 * Parity pinning: the reference cannot be compiled here (no Rust toolchain), so
 * this restatement is pinned against every known-answer test the reference holds
 * for the path (basis/quadrature/element/CG/Jacobi/LU/mesh-generator unit tests,
 * the curved-element test, the shape-function benchmarks and the analytic
 * thermal / patch-test solutions); see tests/test_oracle_pins.py.
 *
 * Every function names the reference lines it follows.  All arrays are
 * row-major; node coordinates are AoS [n][3]; connectivity is [E][10] int64.
 */
#ifndef GEOFEM_ORACLE_H
#define GEOFEM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_mesh orc_mesh;
typedef struct orc_csr orc_csr;

typedef struct {
    int64_t iterations;
    double residual_norm;
    double relative_residual;
    int32_t converged;
    double solve_time;
} orc_stats;

/* ---- mesh generator: mesh_generator_improved.rs:19-169 (HashMap edge cache) ---- */
orc_mesh* orc_generate_cube(int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz);
int64_t orc_mesh_num_nodes(const orc_mesh* m);
int64_t orc_mesh_num_elements(const orc_mesh* m);
void orc_mesh_copy(const orc_mesh* m, double* xyz, int64_t* conn);
void orc_mesh_free(orc_mesh* m);

/* ---- basis / quadrature: basis.rs:56-276, 352-361; quadrature.rs:13-103 ---- */
void orc_shape_functions(const double L[4], double N[10]);
void orc_shape_derivatives_barycentric(const double L[4], double dN[40]);
void orc_jacobian(const double L[4], const double nodes[30], double J[9]);
double orc_det3(const double J[9]);
int orc_shape_derivatives_cartesian(const double L[4], const double nodes[30], double dNdx[30]);
double orc_element_volume(const double nodes[30]);
/* rule: 1, 4, 5 or 11 points; returns number of points written */
int orc_quadrature(int rule, double pts[44], double w[11]);

/* ---- element matrices: element.rs:23-140 and the mechanics element files ---- */
int orc_thermal_stiffness(const double nodes[30], double k, double Ke[100]);
int orc_thermal_mass(const double nodes[30], double rho, double cp, double Me[100]);
int orc_thermal_load(const double nodes[30], double Q, double fe[10]);
void orc_constitutive_matrix(double E, double nu, double D[36]);
void orc_b_matrix(const double dNdx[30], double B[180]);
int orc_elasticity_stiffness(const double nodes[30], double E, double nu, double Ke[900]);
/* element.rs:23-61 for every element of a mesh (OpenMP over elements, as the
 * rayon loop of assembly.rs:69-117): Ke[e][10][10]; k_e per element, or k when
 * k_e is NULL. Returns 0 on a singular Jacobian. */
int orc_thermal_stiffness_all(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn,
                              const double* k_e, double k, double* Ke);
int orc_gravity_load(const double nodes[30], double rho, const double g[3], double fe[30]);

/* ---- assembly: assembly.rs:22-230, 389-437, 906-937 ---- */
/* k_e: per-element conductivity (NULL -> uniform k); parallel != 0 uses the
 * OpenMP element loop + serial triplet merge of the _parallel variant.        */
orc_csr* orc_assemble_thermal_stiffness(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                        const int64_t* conn, const double* k_e, double k,
                                        int parallel);
/* Same CSR, assembled row-parallel (OpenMP) through a node -> element map. */
orc_csr* orc_assemble_thermal_stiffness_rows(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                             const int64_t* conn, const double* k_e, double k);
void orc_assemble_thermal_load(int64_t n_nodes, const double* xyz, int64_t n_elem,
                               const int64_t* conn, double Q, double* f);
orc_csr* orc_assemble_elasticity_stiffness(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                           const int64_t* conn, const double* E_e, double E,
                                           double nu, int parallel);
void orc_assemble_gravity_load(int64_t n_nodes, const double* xyz, int64_t n_elem,
                               const int64_t* conn, double rho, const double g[3], double* f);
/* dirichlet_mask[n] (0/1) and values[n] per DOF (dof.rs:113-140)            */
orc_csr* orc_apply_dirichlet_bcs(const orc_csr* K, const double* f, const uint8_t* dirichlet_mask,
                                 const double* dirichlet_values, double* f_out);
double orc_char_diag(const orc_csr* K);
/* Same result as orc_apply_dirichlet_bcs, row-parallel. */
orc_csr* orc_apply_dirichlet_bcs_rows(const orc_csr* K, const double* f, const uint8_t* dirichlet_mask,
                                      const double* dirichlet_values, double* f_out);

/* ---- sparse matrices (sprs TriMat::to_csr semantics) ---- */
orc_csr* orc_csr_from_triplets(int64_t n_rows, int64_t n_cols, int64_t n_trip, const int64_t* rows,
                               const int64_t* cols, const double* vals);
orc_csr* orc_csr_wrap(int64_t n_rows, int64_t n_cols, const int64_t* indptr, const int32_t* indices,
                      const double* data);
int64_t orc_csr_rows(const orc_csr* A);
int64_t orc_csr_nnz(const orc_csr* A);
void orc_csr_copy(const orc_csr* A, int64_t* indptr, int64_t* indices, double* data);
void orc_csr_apply(const orc_csr* A, const double* x, double* y);
void orc_csr_free(orc_csr* A);

/* ---- solvers: iterative.rs:46-131, preconditioner.rs:37-72, direct.rs:28-73 ---- */
/* iterative.rs:177-278 (BiCGSTAB) and :333-456 (GMRES(restart)), same stats as orc_cg_solve */
void orc_bicgstab_solve(const orc_csr* A, const double* b, int64_t max_iterations, double tolerance,
                        double abs_tolerance, int use_preconditioner, double* x_out, orc_stats* st);
void orc_gmres_solve(const orc_csr* A, const double* b, int64_t max_iterations, int64_t restart, double tolerance,
                     double abs_tolerance, int use_preconditioner, double* x_out, orc_stats* st);
void orc_cg_solve(const orc_csr* A, const double* b, int64_t max_iterations, double tolerance,
                  double abs_tolerance, int use_preconditioner, double* x, orc_stats* stats);
int orc_lu_solve(const orc_csr* A, const double* b, double* x, orc_stats* stats);

/* ---- adjoint checker (no reference counterpart): per-element
 *      g_e = -lambda_e^T K_e u_e, with lambda already zero on Dirichlet DOFs -- */
void orc_thermal_element_gradient(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                  const int64_t* conn, const double* k_e, const double* u,
                                  const double* lam, double* g);
void orc_elasticity_element_gradient(int64_t n_nodes, const double* xyz, int64_t n_elem,
                                     const int64_t* conn, const double* E_e, double nu,
                                     const double* u, const double* lam, double* g);

/* ---- Neumann boundary: fem/boundary.rs:89-266, assembly.rs:248-309 ---- */
void orc_face_nodes(const int64_t elem[10], int local_face, int64_t out[6]);
double orc_face_area(const double coords[18]);
void orc_face_flux(const double coords[18], double flux, double f[6]);
int64_t orc_find_boundary_faces(int64_t n_elem, const int64_t* conn, const uint8_t* node_mask, int64_t* faces);
void orc_apply_neumann_bcs(const double* xyz, const int64_t* conn, int64_t n_faces, const int64_t* faces,
                           const double* flux, double* f);

/* ---- Maxwell viscoelasticity: mechanics/element.rs:257-296, assembly.rs:959-1020,
 *      mechanics/stress_update.rs:39-143 ---- */
int orc_maxwell_history_force(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn,
                              const double* stress, double* f);
int orc_update_stresses_maxwell(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, double E,
                                double nu, double mu, const double* u_n, const double* u_next, double dt,
                                const double* stress_n, double* stress_next);

/* ---- VTU output: mesh/vtk_writer.rs:104-265 with Rust's `{}` for f64 (oracle/vtu.cpp) ---- */
/* Rust Display of one f64 into out (NUL-terminated); returns its length, -1 if cap is too small. */
int orc_format_f64(double v, char* out, int cap);
/* The whole file; returns its size and copies it to out when cap suffices. conn is [E][10]. */
int64_t orc_write_vtu(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, int n_point,
                      const char* const* p_names, const double* const* p_data, const int64_t* p_counts,
                      const int32_t* p_comps, int n_cell, const char* const* c_names, const double* const* c_data,
                      const int64_t* c_counts, const int32_t* c_comps, char* out, int64_t cap);

/* VtkWriter::write (vtk_writer.rs:13-101) and write_nodal_vtu (:531-789); same arguments as orc_write_vtu. */
int64_t orc_write_vtk(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, int n_point,
                      const char* const* p_names, const double* const* p_data, const int64_t* p_counts,
                      const int32_t* p_comps, int n_cell, const char* const* c_names, const double* const* c_data,
                      const int64_t* c_counts, const int32_t* c_comps, char* out, int64_t cap);
int64_t orc_write_vtu_nodal(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, int n_point,
                            const char* const* p_names, const double* const* p_data, const int64_t* p_counts,
                            const int32_t* p_comps, int n_cell, const char* const* c_names,
                            const double* const* c_data, const int64_t* c_counts, const int32_t* c_comps, char* out,
                            int64_t cap);

#ifdef __cplusplus
}
#endif
#endif
