/*
 * geo_fem.h -- C ABI of the B200 (sm_100a) Tet10 FEM hot path.
 *
 * Drop-in for the Rust hot path of msahamed/geo_simulator:
 *   src/fem/element.rs, src/fem/assembly.rs, the src/mechanics/ element, strain,
 *   constitutive and body-force files, src/linalg/{solver,iterative,preconditioner}.rs.
 * Each entry point names the reference item it replaces (file:line inside the
 * reference project). A Rust crate binds these with `extern "C"`; the
 * Python host package (geo_simulator_b200) and include/geofem.hpp bind them too.
 *
 * Conventions
 *  - Every call returns an int status (GEO_OK = 0). Panics of the reference
 *    (singular Jacobian, wrong DOFs per node, failed LU) become error codes;
 *    geo_last_error(ctx) gives the message. Non-convergence is GEO_NOT_CONVERGED
 *    with the solution and statistics still written (the reference reports it
 *    in SolverStats.converged only).
 *  - Pointer arguments to numeric arrays may be host memory (pageable or pinned)
 *    or device memory of the context's GPU: the library checks each pointer and
 *    copies host data in/out itself. All work runs on the context's stream and
 *    every call synchronises before it returns.
 *  - Objects (mesh, dofs, csr, op) are owned by the caller and freed with the
 *    matching *_destroy. One context per host thread; calls on one context are
 *    not re-entrant.
 *  - Indices: connectivity and CSR column indices are int32 (the reference uses
 *    usize); node and DOF counts must stay below 2^31. CSR row pointers are int64.
 *  - Layouts follow the reference: coordinates AoS [n_nodes][3] double,
 *    connectivity [n_elem][10] with the Tet10 local order
 *    [v0 v1 v2 v3 e01 e12 e20 e03 e13 e23] (src/mesh/topology.rs:1-16),
 *    DOF numbering dof = node * dofs_per_node + component (src/fem/dof.rs:87-91).
 */
#ifndef GEO_FEM_H
#define GEO_FEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define GEO_OK 0
#define GEO_ERR_INVALID_ARG 1
#define GEO_ERR_SINGULAR_JACOBIAN 2 /* basis.rs:247 `expect("Singular Jacobian")` */
#define GEO_NOT_CONVERGED 3         /* x and stats valid, stats.converged == 0   */
#define GEO_ERR_BREAKDOWN 4         /* |p^T A p| < 1e-30 (iterative.rs:85); x valid */
#define GEO_ERR_TIMEOUT 5           /* a bounded device-side wait ran out        */
#define GEO_ERR_CUDA 6
#define GEO_ERR_UNSUPPORTED 7
#define GEO_ERR_NO_DEVICE 8
#define GEO_ERR_OUT_OF_MEMORY 9
#define GEO_ERR_SINGULAR_MATRIX 10   /* direct.rs:52 `expect("LU solve failed")` */

/* precision of the matrix-free solver (geo_cg_opts.precision) */
#define GEO_PRECISION_FP64 0  /* plain FP64 throughout (the drop-in semantics)           */
#define GEO_PRECISION_MIXED 1 /* FP32 apply + FP32 PCG, FP64 residual refresh and update */

typedef struct geo_ctx geo_ctx;
typedef struct geo_mesh geo_mesh;
typedef struct geo_dofs geo_dofs;
typedef struct geo_csr geo_csr;
typedef struct geo_op geo_op;

/* ConjugateGradient builder state, iterative.rs:7-44 (defaults :16-24). */
typedef struct geo_cg_opts {
    int64_t max_iterations;     /* with_max_iterations, default 1000  */
    double tolerance;           /* with_tolerance, default 1e-8       */
    double abs_tolerance;       /* with_abs_tolerance, default 1e-12  */
    int32_t use_preconditioner; /* with_preconditioner, default 1 (Jacobi) */
    int32_t precision;          /* matrix-free only: GEO_PRECISION_*, default FP64 */
    double reliable_delta;      /* MIXED: refresh the FP64 residual each time the FP32
                                   residual drops by this factor (default 0.1) */
    double timeout_seconds;     /* bound on every device-side grid barrier (default 10) */
} geo_cg_opts;

/* SolverStats, linalg/solver.rs:5-20, field by field, plus extensions. */
typedef struct geo_solver_stats {
    int64_t iterations;       /* completed PCG iterations (iterative.rs:81-110 counting) */
    double residual_norm;     /* FP64: last recursive ||r||; MIXED: last true ||b - A x|| */
    double relative_residual; /* residual_norm / ||b|| (0 if ||b|| <= 1e-20)       */
    int32_t converged;
    double solve_time;        /* seconds, CUDA events around the device work       */
    /* extensions */
    int32_t status;                 /* GEO_* code of the solve                      */
    int64_t fp64_residual_updates;  /* MIXED: number of FP64 residual refreshes     */
    double b_norm;
    double kernel_time;             /* seconds of device work of the solve (CUDA events) */
    int64_t kernel_launches;        /* kernels the solve launched                   */
} geo_solver_stats;

/* ------------------------------------------------------------------ context */
int geo_device_count(int* count);
int geo_ctx_create(int device, geo_ctx** out);
int geo_ctx_destroy(geo_ctx* ctx);
const char* geo_last_error(const geo_ctx* ctx);
const char* geo_version(void);
/* No counterpart in the reference. Device memory of destroyed objects and finished
 * calls is kept by the library and reused by later calls of the same sizes (freed
 * only after the device has finished the work queued before). This returns the
 * kept memory of every device to the driver; geo_ctx_destroy does so for its
 * device, and an allocation that runs out of memory does so before retrying. */
int geo_release_cached_memory(void);
/* No counterpart in the reference. Counters of the library's device allocator:
 * bytes handed out and not yet freed, bytes kept for reuse, and the number of
 * cudaMalloc calls it has made since the process started (any pointer may be NULL). */
int geo_device_memory_stats(int64_t* live_bytes, int64_t* cached_bytes, int64_t* cuda_mallocs);
int geo_sm_count(const geo_ctx* ctx, int* sm_count);
/* The context's CUDA stream (cudaStream_t), so callers can order or time their
 * own work against the library's launches. */
int geo_ctx_stream(const geo_ctx* ctx, void** stream);

/* ------------------------------------------------------------------ mesh */
/* ImprovedMeshGenerator::generate_cube, mesh_generator_improved.rs:19-169 (host
 * code, bit-exact node numbering and connectivity). geo_generate_cube_size gives
 * the array sizes; xyz is [n_nodes][3], conn is [n_elem][10] (host memory).     */
int geo_generate_cube_size(int64_t nx, int64_t ny, int64_t nz, int64_t* n_nodes, int64_t* n_elem);
int geo_generate_cube(int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz,
                      double* xyz, int32_t* conn);

/* Mesh{geometry.nodes, connectivity.tet10_elements}, mesh/geometry.rs:41-71.
 * Uploaded once; the device keeps SoA coordinates and SoA connectivity.       */
int geo_mesh_create(geo_ctx* ctx, int64_t n_nodes, const double* xyz, int64_t n_elem,
                    const int32_t* conn, geo_mesh** out);
int geo_mesh_destroy(geo_mesh* mesh);

/* ImprovedMeshGenerator::generate_cube, mesh_generator_improved.rs:19-169, run
 * on the device: builds the device mesh directly (no host arrays, no upload)
 * with the node numbering, coordinates and connectivity of geo_generate_cube,
 * bit for bit. The reference returns a host Mesh; geo_mesh_download gives that. */
int geo_mesh_generate_cube(geo_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz,
                           geo_mesh** out);
/* Node and element counts of a device mesh (Mesh::num_nodes / num_elements,
 * mesh/geometry.rs). Either pointer may be NULL.                               */
int geo_mesh_size(const geo_mesh* mesh, int64_t* n_nodes, int64_t* n_elem);
/* Copies a device mesh out in the layout of geo_generate_cube: xyz[n_nodes][3]
 * and conn[n_elem][10], host or device memory; either may be NULL.             */
int geo_mesh_download(const geo_mesh* mesh, double* xyz, int32_t* conn);

/* ------------------------------------------------------------------ VTU output */
/* A point or cell field of VtkWriter::write_vtu (mesh/fields.rs ScalarField /
 * VectorField). components 1: count values; components 3: count [x y z]
 * triples (VectorField::from_dof_vector layout). data is host or device
 * memory; name is written verbatim into Name="...".                            */
typedef struct geo_vtu_field {
    const char* name;
    const double* data;
    int64_t count;
    int32_t components;
} geo_vtu_field;

/* VtkWriter::write_vtu, mesh/vtk_writer.rs:104-265, byte for byte: the ASCII
 * VTU text of the mesh and its fields, formatted on the GPU (every f64 as Rust's
 * `{}`: shortest round-trip digits, positional). Scalar fields are written
 * before vector fields, each in the order given (the reference's two loops over
 * its field maps). *size receives the byte count; with out == NULL nothing is
 * written, otherwise out (host or device memory) must hold capacity >= *size
 * bytes, else GEO_ERR_INVALID_ARG with *size still set.                       */
int geo_vtu_render(geo_ctx* ctx, const geo_mesh* mesh, const geo_vtu_field* point_fields, int32_t n_point,
                   const geo_vtu_field* cell_fields, int32_t n_cell, char* out, int64_t capacity, int64_t* size);
/* The same text streamed to the file `path` (created or truncated); size may be NULL. */
int geo_write_vtu(geo_ctx* ctx, const geo_mesh* mesh, const geo_vtu_field* point_fields, int32_t n_point,
                  const geo_vtu_field* cell_fields, int32_t n_cell, const char* path, int64_t* size);

/* The reference's other writers with the same fields and sinks, selected by format:
 * GEO_VTK_LEGACY    VtkWriter::write, mesh/vtk_writer.rs:13-101 (legacy ASCII .vtk);
 * GEO_VTK_XML       VtkWriter::write_vtu (as geo_vtu_render / geo_write_vtu);
 * GEO_VTK_XML_NODAL VtkWriter::write_nodal_vtu, :531-789 (the builder's default):
 *                   vector point fields one per line, scalar point fields, then
 *                   the named cell fields PlasticStrain, Stress_II, StrainRate_II,
 *                   Pressure, Viscosity, IsYielding, YieldStress, PlasticViscosity
 *                   and SoftenedCohesion summed to the nodes in element order,
 *                   divided by the node's element count only when PlasticStrain
 *                   is present, zero when absent; no CellData.              */
#define GEO_VTK_LEGACY 0
#define GEO_VTK_XML 1
#define GEO_VTK_XML_NODAL 2
int geo_vtk_render(geo_ctx* ctx, const geo_mesh* mesh, int32_t format, const geo_vtu_field* point_fields,
                   int32_t n_point, const geo_vtu_field* cell_fields, int32_t n_cell, char* out, int64_t capacity,
                   int64_t* size);
int geo_write_vtk(geo_ctx* ctx, const geo_mesh* mesh, int32_t format, const geo_vtu_field* point_fields,
                  int32_t n_point, const geo_vtu_field* cell_fields, int32_t n_cell, const char* path, int64_t* size);

/* DofManager::new + set_dirichlet, dof.rs:37-50, :113-130. dirichlet_mask[n_dofs]
 * (nonzero = constrained) and dirichlet_values[n_dofs]; either may be NULL.     */
int geo_dofs_create(geo_ctx* ctx, int64_t n_nodes, int32_t dofs_per_node,
                    const uint8_t* dirichlet_mask, const double* dirichlet_values, geo_dofs** out);
int geo_dofs_num_dirichlet(const geo_dofs* dofs, int64_t* count);
int geo_dofs_destroy(geo_dofs* dofs);

/* ------------------------------------------------------------------ K1: element integration */
/* Per-element matrices for every element of the mesh, row-major per element.
 * k_e / E_e: per-element coefficient array, or NULL for the uniform scalar.   */
/* ElementMatrix::thermal_stiffness, element.rs:23-61 (4-point rule): ke[n_elem][10][10] */
int geo_element_thermal_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const double* k_e, double k,
                                  double* ke);
/* ElementMatrix::thermal_mass, element.rs:74-105 (5-point rule): me[n_elem][10][10] */
int geo_element_thermal_mass(geo_ctx* ctx, const geo_mesh* mesh, double density,
                             double specific_heat, double* me);
/* ElementMatrix::thermal_load, element.rs:117-140: fe[n_elem][10] */
int geo_element_thermal_load(geo_ctx* ctx, const geo_mesh* mesh, double source, double* fe);
/* ElasticityElement::stiffness_matrix, mechanics/element.rs:33-65 with
 * IsotropicElasticity::constitutive_matrix, mechanics/constitutive.rs:63-102:
 * ke[n_elem][30][30] */
int geo_element_elasticity_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const double* E_e,
                                     double E, double nu, double* ke);
/* BodyForce::gravity_load, mechanics/body_force.rs:49-84: fe[n_elem][30] */
int geo_element_gravity_load(geo_ctx* ctx, const geo_mesh* mesh, double density,
                             const double gravity[3], double* fe);

/* ------------------------------------------------------------------ K2/K3: CSR assembly */
/* Assembler::assemble_thermal_stiffness_parallel, assembly.rs:69-117. Rows and
 * columns are node ids (dofs must have 1 DOF per node). Structure bit-exact with
 * sprs TriMat::to_csr: sorted columns, duplicates summed (in element order),
 * every structural entry kept.                                                 */
int geo_assemble_thermal_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs,
                                   const double* k_e, double k, geo_csr** K);
/* Assembler::assemble_thermal_load, assembly.rs:130-154: f[n_dofs] */
int geo_assemble_thermal_load(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs,
                              double source, double* f);
/* Assembler::apply_dirichlet_bcs, assembly.rs:168-230: char_diag = max(1, max|K_ii|);
 * free rows: f_i -= sum_{j in D} K_ij g_j and D columns dropped; D rows: char_diag
 * on the diagonal, f_i = g_i * char_diag.                                      */
int geo_apply_dirichlet_bcs(geo_ctx* ctx, const geo_csr* K, const double* f, const geo_dofs* dofs,
                            geo_csr** K_bc, double* f_bc);
/* Assembler::assemble_elasticity_stiffness_parallel, assembly.rs:389-437
 * (GEO_ERR_INVALID_ARG unless 3 DOFs per node, as the reference's assert at :394). */
int geo_assemble_elasticity_stiffness(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs,
                                      const double* E_e, double E, double nu, geo_csr** K);
/* Assembler::assemble_gravity_load, assembly.rs:906-937 */
int geo_assemble_gravity_load(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs,
                              double density, const double gravity[3], double* f);

/* ------------------------------------------------------------------ Neumann (flux) boundary */
/* Faces are (element, local face) int32 pairs; local face f is the face opposite
 * vertex f, with the 6 nodes of Tet10Face::from_element_face (boundary.rs:89-130).
 * Per-face flux: flux_f[n_faces], or NULL for the uniform scalar flux.          */
/* Tet10Face::integrate_flux (boundary.rs:202-266) for many faces: fe[n_faces][6] */
int geo_face_flux(geo_ctx* ctx, const geo_mesh* mesh, int64_t n_faces, const int32_t* faces,
                  const double* flux_f, double flux, double* fe);
/* Tet10Face::area (boundary.rs:136-196): area[n_faces] */
int geo_face_area(geo_ctx* ctx, const geo_mesh* mesh, int64_t n_faces, const int32_t* faces, double* area);
/* Assembler::find_boundary_faces (assembly.rs:287-309) with the condition evaluated
 * per node by the caller: node_mask[n_nodes] != 0 where it holds. Writes the faces
 * whose 6 nodes all satisfy it, in (element, local face) order, and their count;
 * faces may be NULL to query the count (capacity max_faces pairs).            */
int geo_find_boundary_faces(geo_ctx* ctx, const geo_mesh* mesh, const uint8_t* node_mask, int64_t max_faces,
                            int32_t* faces, int64_t* n_faces);
/* Assembler::apply_neumann_bcs (assembly.rs:248-274): f[node] += face flux
 * contributions (f indexed by node id, n_f >= n_nodes, updated in place). The
 * sum per node runs in face order (deterministic).                             */
int geo_apply_neumann_bcs(geo_ctx* ctx, const geo_mesh* mesh, int64_t n_faces, const int32_t* faces,
                          const double* flux_f, double flux, int64_t n_f, double* f);

/* ------------------------------------------------------------------ Maxwell viscoelasticity */
/* Element stresses are Voigt 6-vectors [xx yy zz xy yz zx] per element (StressHistory,
 * mesh/state.rs:12-75), stress[n_elem][6]. Material: E > 0, nu in (-1, 0.5), mu > 0
 * (MaxwellViscoelasticity::new, mechanics/constitutive.rs:317-329).               */
/* The history force of assemble_maxwell_viscoelastic_parallel (assembly.rs:959-1020):
 * f[3 n_nodes] = -sum_e sum_q w |det J| B^T sigma_e (mechanics/element.rs:257-296). */
int geo_maxwell_history_force(geo_ctx* ctx, const geo_mesh* mesh, const double* stress, double* f);
/* Assembler::assemble_maxwell_viscoelastic_parallel (assembly.rs:959-1020): the elastic
 * stiffness (as geo_assemble_elasticity_stiffness with E, nu) and the history force. */
int geo_assemble_maxwell_viscoelastic(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs, double E,
                                      double nu, double mu, double dt, const double* stress, geo_csr** K,
                                      double* f_history);
/* update_stresses_maxwell (mechanics/stress_update.rs:39-143): stress_next[n_elem][6]
 * from the strain increment of u_next - u_n averaged over the 4 points, elastic
 * predictor, deviatoric part relaxed by 1 / (1 + dt / tau_M).                    */
int geo_update_stresses_maxwell(geo_ctx* ctx, const geo_mesh* mesh, double E, double nu, double mu,
                                const double* u_n, const double* u_next, double dt, const double* stress_n,
                                double* stress_next);

/* sprs CsMat<f64> stand-in (device resident). */
int geo_csr_create(geo_ctx* ctx, int64_t n_rows, int64_t n_cols, int64_t nnz, const int64_t* indptr,
                   const int32_t* indices, const double* data, geo_csr** out);
int geo_csr_info(const geo_csr* A, int64_t* n_rows, int64_t* n_cols, int64_t* nnz);
int geo_csr_copy(const geo_csr* A, int64_t* indptr, int32_t* indices, double* data);
int geo_csr_device_ptrs(const geo_csr* A, const int64_t** indptr, const int32_t** indices,
                        const double** data);
/* impl LinearOperator for CsMat<f64>, linalg/solver.rs:61-73: y = A x */
int geo_csr_apply(geo_ctx* ctx, const geo_csr* A, const double* x, double* y);
int geo_csr_destroy(geo_csr* A);

/* ------------------------------------------------------------------ K4: FP64 Jacobi-PCG */
void geo_cg_opts_default(geo_cg_opts* opts);
/* ConjugateGradient::solve, iterative.rs:123-131 -> solve_with_operator_internal
 * :46-119 with JacobiPreconditioner::new, preconditioner.rs:37-51. x0 = 0; stops when
 * ||r|| < tol ||b|| or ||r|| < abs_tol; returns zeros when ||b|| < 1e-25.
 * One persistent kernel runs the whole solve.                                  */
int geo_cg_solve(geo_ctx* ctx, const geo_csr* A, const double* b, const geo_cg_opts* opts,
                 double* x, geo_solver_stats* stats);

/* BiCGSTAB::solve (linalg/iterative.rs:150-301) and GMRES::solve (:303-479), the
 * CG drop-in's siblings: FP64 on the assembled CSR, right-preconditioned with the
 * Jacobi inverse diagonal (opts->use_preconditioner) or the identity, with the
 * reference's stopping rules and iteration counting (GMRES counts Arnoldi steps).
 * opts: max_iterations, tolerance, abs_tolerance, use_preconditioner and
 * timeout_seconds are used. Returns GEO_NOT_CONVERGED or GEO_ERR_BREAKDOWN (a
 * |denominator| < 1e-40 in BiCGSTAB) with x and stats valid, as geo_cg_solve.
 * restart: the GMRES cycle length, 1..64 (the reference's default is 10).      */
int geo_bicgstab_solve(geo_ctx* ctx, const geo_csr* A, const double* b, const geo_cg_opts* opts, double* x,
                       geo_solver_stats* stats);
int geo_gmres_solve(geo_ctx* ctx, const geo_csr* A, const double* b, const geo_cg_opts* opts, int32_t restart,
                    double* x, geo_solver_stats* stats);

/* DirectSolver::solve (linalg/direct.rs:28-73): the CSR matrix densified on the
 * device and solved by LU with partial pivoting (first row of largest |a_ik|, as
 * the reference's dense LU), FP64, in one persistent cooperative kernel.
 * n_rows <= 16384 (the dense factor takes 8 n^2 bytes; else GEO_ERR_INVALID_ARG).
 * A zero pivot returns GEO_ERR_SINGULAR_MATRIX (the reference panics, "LU solve
 * failed"). stats: iterations 0, residual_norm ||b - A x||, relative_residual
 * (solver.rs:165-175), converged = relative_residual < 1e-8 (direct.rs:58-66). */
int geo_direct_solve(geo_ctx* ctx, const geo_csr* A, const double* b, double* x, geo_solver_stats* stats);

/* No counterpart in the reference. geo_cg_solve without any device allocation, for
 * callers that must not call cudaMalloc/cudaFree between solves (device memory
 * held by another allocator; loops that cannot take cudaFree's device-wide sync).
 * Same kernel and results as geo_cg_solve. Work vectors come from one static
 * device array per device (8.25 MiB), so: n_rows <= GEO_NOALLOC_MAX_ROWS (else
 * GEO_ERR_INVALID_ARG); b_dev and x_dev must be device memory on the context's
 * device; calls that overlap on one device race on the array and must be
 * serialised; the first call on a device looks the array up (the runtime may load
 * the module then), so make it before the allocation-free phase and before any
 * stream capture. The barrier word and result slot are zeroed before each launch. */
#define GEO_NOALLOC_MAX_ROWS 262144
int geo_cg_solve_noalloc(geo_ctx* ctx, const geo_csr* A, const double* b_dev, const geo_cg_opts* opts,
                         double* x_dev, geo_solver_stats* stats);

/* ------------------------------------------------------------------ K5/K6: matrix-free */
/* Matrix-free Dirichlet-eliminated operator K_bc of the thermal problem (the
 * operator apply_dirichlet_bcs(assemble_thermal_stiffness_parallel(..)) builds,
 * assembly.rs:69-117 + :168-230) or of 3-DOF elasticity (assembly.rs:389-437).
 * Replaces the Solver::solve_with_operator seam, linalg/solver.rs:112-120.     */
int geo_thermal_operator_create(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs,
                                const double* k_e, double k, geo_op** out);
int geo_elasticity_operator_create(geo_ctx* ctx, const geo_mesh* mesh, const geo_dofs* dofs,
                                   const double* E_e, double E, double nu, geo_op** out);
/* Replace the per-element coefficients (k_e or E_e; NULL -> uniform scalar). */
int geo_op_set_coefficients(geo_op* op, const double* coef_e, double coef);
int geo_op_info(const geo_op* op, int64_t* n_dofs, int64_t* n_elem, double* char_diag);
/* y = K_bc x (LinearOperator::apply, linalg/solver.rs:41-58); precision FP64 or MIXED
 * (MIXED applies the FP32 operator to the FP32-rounded x). */
int geo_op_apply(geo_op* op, const double* x, double* y, int32_t precision);
/* The vector half of apply_dirichlet_bcs (assembly.rs:195-218), matrix-free. */
int geo_op_lift_rhs(geo_op* op, const double* f, double* f_bc);
/* diag(K_bc), the Jacobi diagonal (preconditioner.rs:37-51). */
int geo_op_diagonal(geo_op* op, double* diag);
/* Jacobi-PCG on K_bc, two kernels per iteration run from CUDA graphs of 16
 * iterations: the patch kernel applies K_bc fused with p = D^-1 r + beta p and the
 * p.Ap reduction; the node kernel does the axpys, r.r and r.z and the stopping
 * test (single-pass grid reductions, scalars resident on the device, no host
 * round trip inside a graph). FP64: the reference's stopping rule on the recursive
 * residual. MIXED: FP32 inner PCG with FP32 accumulation; the FP64 residual
 * b - A x and the FP64 solution update are refreshed on device whenever the FP32
 * residual fell by opts.reliable_delta; convergence is decided on the FP64 residual. */
int geo_cg_solve_matfree(geo_op* op, const double* b, const geo_cg_opts* opts, double* x,
                         geo_solver_stats* stats);

/* ------------------------------------------------------------------ K7: adjoint (vjp) */
/* Per-element g_e = -lambda_e^T K_e u_e, lambda zeroed on Dirichlet DOFs. For the
 * thermal operator this is dJ/d(ln k_e); for elasticity dJ/d(ln E_e).        */
int geo_op_element_gradient(geo_op* op, const double* u, const double* lambda, double* grad_e);
/* forward: u = K_bc^{-1} lift(f)  (apply_dirichlet_bcs + ConjugateGradient::solve) */
int geo_forward(geo_op* op, const double* f, const geo_cg_opts* opts, double* u,
                geo_solver_stats* stats);
/* backward (vector-Jacobian product): given dJ/du, solve K_bc lambda = dJ/du (free
 * rows) and return dJ/d(ln coef_e). u may be NULL: the forward solution is then
 * recomputed from f (recompute instead of store).                             */
int geo_vjp(geo_op* op, const double* f, const double* u, const double* dJ_du,
            const geo_cg_opts* opts, double* dJ_dlncoef, geo_solver_stats* stats);
/* Diagnostic, no reference counterpart: average device time (ms) of the two kernels
 * of one matrix-free PCG iteration -- the patch kernel in PCG mode and the node
 * update -- over `iterations` (1..4096) iterations started from b (original
 * numbering, host or device), with the stopping tests disabled so that every
 * launch does full work. CUDA events between the launches on the context stream. */
int geo_op_time_pcg_kernels(geo_op* op, const double* b, int32_t precision, int32_t iterations,
                            double* patch_ms, double* update_ms);
int geo_op_destroy(geo_op* op);

/* ------------------------------------------------------------------ failure detection */
/* Launches a persistent kernel whose block 0 skips one grid barrier on purpose so
 * that every other block's bounded wait runs out after timeout_seconds; returns
 * GEO_ERR_TIMEOUT when the device-side timeout fired and the context stays usable. */
int geo_debug_barrier_timeout(geo_ctx* ctx, double timeout_seconds);

#ifdef __cplusplus
}
#endif
#endif /* GEO_FEM_H */
