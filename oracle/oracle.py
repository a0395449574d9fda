"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of bench.py
import this module, and only as the checker. The product package
(geo_simulator_b200) never imports it.

Every wrapper returns numpy arrays; connectivity is ``int64 [E, 10]`` and
coordinates ``float64 [N, 3]`` as in the reference's ``Mesh``
(src/mesh/geometry.rs:8-71, src/mesh/topology.rs:13-86).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build() -> str:
    """Compile oracle/liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class OrcStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("residual_norm", C.c_double),
                ("relative_residual", C.c_double), ("converged", C.c_int32),
                ("solve_time", C.c_double)]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_U8 = C.POINTER(C.c_uint8)


def _declare(L):
    sig = {
        "orc_generate_cube": (_P, [C.c_int64] * 3 + [C.c_double] * 3),
        "orc_mesh_num_nodes": (C.c_int64, [_P]),
        "orc_mesh_num_elements": (C.c_int64, [_P]),
        "orc_mesh_copy": (None, [_P, _D, _I64]),
        "orc_mesh_free": (None, [_P]),
        "orc_shape_functions": (None, [_D, _D]),
        "orc_shape_derivatives_barycentric": (None, [_D, _D]),
        "orc_jacobian": (None, [_D, _D, _D]),
        "orc_det3": (C.c_double, [_D]),
        "orc_shape_derivatives_cartesian": (C.c_int, [_D, _D, _D]),
        "orc_element_volume": (C.c_double, [_D]),
        "orc_quadrature": (C.c_int, [C.c_int, _D, _D]),
        "orc_thermal_stiffness": (C.c_int, [_D, C.c_double, _D]),
        "orc_thermal_stiffness_all": (C.c_int, [C.c_int64, _D, C.c_int64, _I64, _D, C.c_double, _D]),
        "orc_thermal_mass": (C.c_int, [_D, C.c_double, C.c_double, _D]),
        "orc_thermal_load": (C.c_int, [_D, C.c_double, _D]),
        "orc_constitutive_matrix": (None, [C.c_double, C.c_double, _D]),
        "orc_b_matrix": (None, [_D, _D]),
        "orc_elasticity_stiffness": (C.c_int, [_D, C.c_double, C.c_double, _D]),
        "orc_gravity_load": (C.c_int, [_D, C.c_double, _D, _D]),
        "orc_assemble_thermal_stiffness": (_P, [C.c_int64, _D, C.c_int64, _I64, _D, C.c_double, C.c_int]),
        "orc_assemble_thermal_stiffness_rows": (_P, [C.c_int64, _D, C.c_int64, _I64, _D, C.c_double]),
        "orc_apply_dirichlet_bcs_rows": (_P, [_P, _D, _U8, _D, _D]),
        "orc_assemble_thermal_load": (None, [C.c_int64, _D, C.c_int64, _I64, C.c_double, _D]),
        "orc_assemble_elasticity_stiffness": (_P, [C.c_int64, _D, C.c_int64, _I64, _D, C.c_double,
                                                   C.c_double, C.c_int]),
        "orc_assemble_gravity_load": (None, [C.c_int64, _D, C.c_int64, _I64, C.c_double, _D, _D]),
        "orc_apply_dirichlet_bcs": (_P, [_P, _D, _U8, _D, _D]),
        "orc_char_diag": (C.c_double, [_P]),
        "orc_csr_from_triplets": (_P, [C.c_int64, C.c_int64, C.c_int64, _I64, _I64, _D]),
        "orc_csr_wrap": (_P, [C.c_int64, C.c_int64, _I64, C.c_void_p, _D]),
        "orc_csr_rows": (C.c_int64, [_P]),
        "orc_csr_nnz": (C.c_int64, [_P]),
        "orc_csr_copy": (None, [_P, _I64, _I64, _D]),
        "orc_csr_apply": (None, [_P, _D, _D]),
        "orc_csr_free": (None, [_P]),
        "orc_cg_solve": (None, [_P, _D, C.c_int64, C.c_double, C.c_double, C.c_int, _D,
                                C.POINTER(OrcStats)]),
        "orc_lu_solve": (C.c_int, [_P, _D, _D, C.POINTER(OrcStats)]),
        "orc_bicgstab_solve": (None, [_P, _D, C.c_int64, C.c_double, C.c_double, C.c_int, _D,
                                      C.POINTER(OrcStats)]),
        "orc_gmres_solve": (None, [_P, _D, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int, _D,
                                   C.POINTER(OrcStats)]),
        "orc_thermal_element_gradient": (None, [C.c_int64, _D, C.c_int64, _I64, _D, _D, _D, _D]),
        "orc_elasticity_element_gradient": (None, [C.c_int64, _D, C.c_int64, _I64, _D, C.c_double,
                                                   _D, _D, _D]),
        "orc_face_nodes": (None, [_I64, C.c_int, _I64]),
        "orc_face_area": (C.c_double, [_D]),
        "orc_face_flux": (None, [_D, C.c_double, _D]),
        "orc_find_boundary_faces": (C.c_int64, [C.c_int64, _I64, _U8, _I64]),
        "orc_apply_neumann_bcs": (None, [_D, _I64, C.c_int64, _I64, _D, _D]),
        "orc_maxwell_history_force": (C.c_int, [C.c_int64, _D, C.c_int64, _I64, _D, _D]),
        "orc_update_stresses_maxwell": (C.c_int, [C.c_int64, _D, C.c_int64, _I64, C.c_double, C.c_double,
                                                  C.c_double, _D, _D, C.c_double, _D, _D]),
        "orc_format_f64": (C.c_int, [C.c_double, C.c_char_p, C.c_int]),
        "orc_write_vtu": (C.c_int64, [C.c_int64, _D, C.c_int64, _I64, C.c_int, C.c_void_p, C.c_void_p, _I64,
                                      C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, _I64, C.c_void_p,
                                      C.c_char_p, C.c_int64]),
        "orc_write_vtk": (C.c_int64, [C.c_int64, _D, C.c_int64, _I64, C.c_int, C.c_void_p, C.c_void_p, _I64,
                                      C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, _I64, C.c_void_p,
                                      C.c_char_p, C.c_int64]),
        "orc_write_vtu_nodal": (C.c_int64, [C.c_int64, _D, C.c_int64, _I64, C.c_int, C.c_void_p, C.c_void_p,
                                            _I64, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, _I64, C.c_void_p,
                                            C.c_char_p, C.c_int64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


# ------------------------------------------------------------------- mesh
def generate_cube(nx, ny, nz, lx, ly, lz):
    """ImprovedMeshGenerator::generate_cube (mesh_generator_improved.rs:19-169)."""
    L = lib()
    h = L.orc_generate_cube(nx, ny, nz, lx, ly, lz)
    n, e = L.orc_mesh_num_nodes(h), L.orc_mesh_num_elements(h)
    xyz = np.empty((n, 3), np.float64)
    conn = np.empty((e, 10), np.int64)
    L.orc_mesh_copy(h, _d(xyz), _i(conn))
    L.orc_mesh_free(h)
    return xyz, conn


# ------------------------------------------------------------------- basis
def shape_functions(L4):
    out = np.empty(10)
    lib().orc_shape_functions(_d(_f64(L4)), _d(out))
    return out


def shape_derivatives_barycentric(L4):
    out = np.empty(40)
    lib().orc_shape_derivatives_barycentric(_d(_f64(L4)), _d(out))
    return out.reshape(10, 4)


def jacobian(L4, nodes):
    out = np.empty(9)
    lib().orc_jacobian(_d(_f64(L4)), _d(_f64(nodes)), _d(out))
    return out.reshape(3, 3)


def det3(J):
    return lib().orc_det3(_d(_f64(J)))


def shape_derivatives_cartesian(L4, nodes):
    out = np.empty(30)
    ok = lib().orc_shape_derivatives_cartesian(_d(_f64(L4)), _d(_f64(nodes)), _d(out))
    if not ok:
        raise ZeroDivisionError("Singular Jacobian")
    return out.reshape(10, 3)


def element_volume(nodes):
    return lib().orc_element_volume(_d(_f64(nodes)))


def quadrature(rule):
    pts, w = np.empty(44), np.empty(11)
    n = lib().orc_quadrature(rule, _d(pts), _d(w))
    return pts[: 4 * n].reshape(n, 4), w[:n].copy()


# ------------------------------------------------------------------- elements
def thermal_stiffness(nodes, k):
    out = np.empty(100)
    if not lib().orc_thermal_stiffness(_d(_f64(nodes)), k, _d(out)):
        raise ZeroDivisionError("Singular Jacobian")
    return out.reshape(10, 10)


def thermal_stiffness_all(xyz, conn, k=1.0, k_e=None):
    """element.rs:23-61 for every element (OpenMP): array [E][10][10]."""
    xyz, conn = _f64(xyz), _i64(conn)
    out = np.empty((conn.shape[0], 10, 10))
    ke = _d(_f64(k_e)) if k_e is not None else None
    if not lib().orc_thermal_stiffness_all(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn), ke, float(k), _d(out)):
        raise ZeroDivisionError("Singular Jacobian")
    return out


def thermal_mass(nodes, rho, cp):
    out = np.empty(100)
    lib().orc_thermal_mass(_d(_f64(nodes)), rho, cp, _d(out))
    return out.reshape(10, 10)


def thermal_load(nodes, Q):
    out = np.empty(10)
    lib().orc_thermal_load(_d(_f64(nodes)), Q, _d(out))
    return out


def constitutive_matrix(E, nu):
    out = np.empty(36)
    lib().orc_constitutive_matrix(E, nu, _d(out))
    return out.reshape(6, 6)


def b_matrix(dNdx):
    out = np.empty(180)
    lib().orc_b_matrix(_d(_f64(dNdx)), _d(out))
    return out.reshape(6, 30)


def elasticity_stiffness(nodes, E, nu):
    out = np.empty(900)
    if not lib().orc_elasticity_stiffness(_d(_f64(nodes)), E, nu, _d(out)):
        raise ZeroDivisionError("Singular Jacobian")
    return out.reshape(30, 30)


def gravity_load(nodes, rho, g):
    out = np.empty(30)
    lib().orc_gravity_load(_d(_f64(nodes)), rho, _d(_f64(g)), _d(out))
    return out


# ------------------------------------------------------------------- CSR
@dataclass
class Csr:
    """Host CSR (sprs CsMat layout): int64 indptr/indices, float64 data."""
    n_rows: int
    n_cols: int
    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    _h: int = 0

    @property
    def nnz(self):
        return int(self.indices.size)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.data, self.indices, self.indptr), shape=(self.n_rows, self.n_cols))

    def handle(self):
        """Re-materialise an oracle-side handle (for CG / LU / Dirichlet)."""
        rows = np.repeat(np.arange(self.n_rows, dtype=np.int64), np.diff(self.indptr))
        return lib().orc_csr_from_triplets(self.n_rows, self.n_cols, self.nnz, _i(rows),
                                           _i(_i64(self.indices)), _d(_f64(self.data)))


def _csr_from_handle(h, n_cols=None):
    L = lib()
    if not h:
        raise ZeroDivisionError("Singular Jacobian")
    n, nnz = L.orc_csr_rows(h), L.orc_csr_nnz(h)
    indptr = np.empty(n + 1, np.int64)
    indices = np.empty(nnz, np.int64)
    data = np.empty(nnz, np.float64)
    L.orc_csr_copy(h, _i(indptr), _i(indices), _d(data))
    L.orc_csr_free(h)
    return Csr(n, n if n_cols is None else n_cols, indptr, indices, data)


def csr_from_triplets(n_rows, n_cols, rows, cols, vals):
    rows, cols, vals = _i64(rows), _i64(cols), _f64(vals)
    h = lib().orc_csr_from_triplets(n_rows, n_cols, rows.size, _i(rows), _i(cols), _d(vals))
    return _csr_from_handle(h, n_cols)


# ------------------------------------------------------------------- assembly
def assemble_thermal_stiffness(xyz, conn, k=1.0, k_e=None, parallel=True):
    """Assembler::assemble_thermal_stiffness_parallel / _serial (assembly.rs:22-117)."""
    xyz, conn = _f64(xyz), _i64(conn)
    ke = _d(_f64(k_e)) if k_e is not None else None
    h = lib().orc_assemble_thermal_stiffness(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn), ke,
                                             float(k), int(bool(parallel)))
    return _csr_from_handle(h)


def assemble_thermal_load(xyz, conn, Q):
    """Assembler::assemble_thermal_load (assembly.rs:130-154)."""
    xyz, conn = _f64(xyz), _i64(conn)
    f = np.empty(xyz.shape[0])
    lib().orc_assemble_thermal_load(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn), Q, _d(f))
    return f


def assemble_elasticity_stiffness(xyz, conn, E=1.0, nu=0.25, E_e=None, parallel=True):
    """Assembler::assemble_elasticity_stiffness_parallel (assembly.rs:389-437)."""
    xyz, conn = _f64(xyz), _i64(conn)
    ee = _d(_f64(E_e)) if E_e is not None else None
    h = lib().orc_assemble_elasticity_stiffness(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn), ee,
                                                float(E), float(nu), int(bool(parallel)))
    return _csr_from_handle(h)


def assemble_gravity_load(xyz, conn, rho, g):
    """Assembler::assemble_gravity_load (assembly.rs:906-937)."""
    xyz, conn = _f64(xyz), _i64(conn)
    f = np.empty(3 * xyz.shape[0])
    lib().orc_assemble_gravity_load(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn), rho,
                                    _d(_f64(g)), _d(f))
    return f


def apply_dirichlet_bcs(K: Csr, f, mask, values):
    """Assembler::apply_dirichlet_bcs (assembly.rs:168-230)."""
    h = K.handle()
    mask = np.ascontiguousarray(mask, dtype=np.uint8)
    fout = np.empty(K.n_rows)
    h2 = lib().orc_apply_dirichlet_bcs(h, _d(_f64(f)), mask.ctypes.data_as(_U8),
                                       _d(_f64(values)), _d(fout))
    lib().orc_csr_free(h)
    return _csr_from_handle(h2, K.n_cols), fout


def char_diag(K: Csr):
    h = K.handle()
    v = lib().orc_char_diag(h)
    lib().orc_csr_free(h)
    return v


def csr_apply(K: Csr, x):
    h = K.handle()
    y = np.empty(K.n_rows)
    lib().orc_csr_apply(h, _d(_f64(x)), _d(y))
    lib().orc_csr_free(h)
    return y


class ThermalSystem:
    """K_bc and f_bc of the thermal problem held on the oracle side (no copies to numpy):
    the row-parallel assembler + Dirichlet pass, then the reference CG on it."""

    def __init__(self, xyz, conn, k_e, Q, mask, values):
        L = lib()
        xyz, conn = _f64(xyz), _i64(conn)
        self.n = xyz.shape[0]
        hk = L.orc_assemble_thermal_stiffness_rows(self.n, _d(xyz), conn.shape[0], _i(conn), _d(_f64(k_e)), 0.0)
        f = np.empty(self.n)
        L.orc_assemble_thermal_load(self.n, _d(xyz), conn.shape[0], _i(conn), Q, _d(f))
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        self.fb = np.empty(self.n)
        self.h = L.orc_apply_dirichlet_bcs_rows(hk, _d(f), mask.ctypes.data_as(_U8), _d(_f64(values)),
                                                _d(self.fb))
        L.orc_csr_free(hk)
        self.nnz = L.orc_csr_nnz(self.h)

    def cg(self, max_iterations, tolerance=1e-8, abs_tolerance=1e-12):
        x = np.empty(self.n)
        st = OrcStats()
        lib().orc_cg_solve(self.h, _d(self.fb), int(max_iterations), tolerance, abs_tolerance, 1, _d(x),
                           C.byref(st))
        return x, st

    def __del__(self):
        try:
            lib().orc_csr_free(self.h)
        except Exception:
            pass


class CsrHandle:
    """Oracle-side copy of a CSR given as (int64 indptr, int32 indices, float64 data)."""

    def __init__(self, n_rows, n_cols, indptr, indices, data):
        indptr = np.ascontiguousarray(indptr, np.int64)
        indices = np.ascontiguousarray(indices, np.int32)
        data = np.ascontiguousarray(data, np.float64)
        self.n_rows = n_rows
        self.h = lib().orc_csr_wrap(n_rows, n_cols, _i(indptr), indices.ctypes.data, _d(data))

    def cg(self, b, max_iterations, tolerance=1e-8, abs_tolerance=1e-12, use_preconditioner=True):
        """The reference loop (iterative.rs:46-119) on this matrix."""
        x = np.empty(self.n_rows)
        st = OrcStats()
        lib().orc_cg_solve(self.h, _d(_f64(b)), int(max_iterations), tolerance, abs_tolerance,
                           int(bool(use_preconditioner)), _d(x), C.byref(st))
        return x, st

    def __del__(self):
        try:
            lib().orc_csr_free(self.h)
        except Exception:
            pass


# ------------------------------------------------------------------- solvers
def cg_solve(A: Csr, b, max_iterations=1000, tolerance=1e-8, abs_tolerance=1e-12,
             use_preconditioner=True):
    """ConjugateGradient::solve (iterative.rs:46-131)."""
    h = A.handle()
    x = np.empty(A.n_rows)
    st = OrcStats()
    lib().orc_cg_solve(h, _d(_f64(b)), int(max_iterations), tolerance, abs_tolerance,
                       int(bool(use_preconditioner)), _d(x), C.byref(st))
    lib().orc_csr_free(h)
    return x, st


def bicgstab_solve(A: Csr, b, max_iterations=1000, tolerance=1e-8, abs_tolerance=1e-12,
                   use_preconditioner=True):
    """BiCGSTAB::solve (iterative.rs:177-278)."""
    h = A.handle()
    x = np.empty(A.n_rows)
    st = OrcStats()
    lib().orc_bicgstab_solve(h, _d(_f64(b)), int(max_iterations), tolerance, abs_tolerance,
                             int(bool(use_preconditioner)), _d(x), C.byref(st))
    lib().orc_csr_free(h)
    return x, st


def gmres_solve(A: Csr, b, max_iterations=1000, restart=10, tolerance=1e-8, abs_tolerance=1e-12,
                use_preconditioner=True):
    """GMRES::solve (iterative.rs:333-456)."""
    h = A.handle()
    x = np.empty(A.n_rows)
    st = OrcStats()
    lib().orc_gmres_solve(h, _d(_f64(b)), int(max_iterations), int(restart), tolerance, abs_tolerance,
                          int(bool(use_preconditioner)), _d(x), C.byref(st))
    lib().orc_csr_free(h)
    return x, st


def lu_solve(A: Csr, b):
    """DirectSolver::solve (direct.rs:28-73)."""
    h = A.handle()
    x = np.empty(A.n_rows)
    st = OrcStats()
    ok = lib().orc_lu_solve(h, _d(_f64(b)), _d(x), C.byref(st))
    lib().orc_csr_free(h)
    if not ok:
        raise np.linalg.LinAlgError("LU solve failed")
    return x, st


# ------------------------------------------------------------------- adjoint checker
def thermal_element_gradient(xyz, conn, k_e, u, lam):
    xyz, conn = _f64(xyz), _i64(conn)
    g = np.empty(conn.shape[0])
    lib().orc_thermal_element_gradient(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn),
                                       _d(_f64(k_e)), _d(_f64(u)), _d(_f64(lam)), _d(g))
    return g


def elasticity_element_gradient(xyz, conn, E_e, nu, u, lam):
    xyz, conn = _f64(xyz), _i64(conn)
    g = np.empty(conn.shape[0])
    lib().orc_elasticity_element_gradient(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn),
                                          _d(_f64(E_e)), float(nu), _d(_f64(u)), _d(_f64(lam)),
                                          _d(g))
    return g


# ------------------------------------------------------------------- Neumann boundary
def face_nodes(elem, local_face):
    """Tet10Face::from_element_face (boundary.rs:89-130)."""
    out = np.empty(6, np.int64)
    lib().orc_face_nodes(_i(_i64(elem)), int(local_face), _i(out))
    return out


def face_area(coords6):
    return lib().orc_face_area(_d(_f64(coords6)))


def face_flux(coords6, flux):
    """Tet10Face::integrate_flux (boundary.rs:202-266)."""
    f = np.empty(6)
    lib().orc_face_flux(_d(_f64(coords6)), float(flux), _d(f))
    return f


def find_boundary_faces(conn, node_mask):
    """Assembler::find_boundary_faces (assembly.rs:287-309) with the condition
    evaluated per node: [(element, local_face)] whose 6 nodes all satisfy it."""
    conn = _i64(conn)
    faces = np.empty((4 * conn.shape[0], 2), np.int64)
    n = lib().orc_find_boundary_faces(conn.shape[0], _i(conn), np.ascontiguousarray(node_mask, np.uint8).ctypes.data_as(_U8), _i(faces))
    return faces[:n].copy()


def apply_neumann_bcs(xyz, conn, faces, flux, f):
    """Assembler::apply_neumann_bcs (assembly.rs:248-274); returns f + face fluxes."""
    xyz, conn, faces = _f64(xyz), _i64(conn), _i64(faces).reshape(-1, 2)
    flux = np.broadcast_to(np.asarray(flux, np.float64), (faces.shape[0],)).copy()
    out = _f64(f).copy()
    lib().orc_apply_neumann_bcs(_d(xyz), _i(conn), faces.shape[0], _i(faces), _d(flux), _d(out))
    return out


# ------------------------------------------------------------------- Maxwell viscoelasticity
def maxwell_history_force(xyz, conn, stress):
    """f_history of assemble_maxwell_viscoelastic_parallel (assembly.rs:959-1020)."""
    xyz, conn = _f64(xyz), _i64(conn)
    f = np.empty(3 * xyz.shape[0])
    assert lib().orc_maxwell_history_force(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn),
                                           _d(_f64(stress)), _d(f)) == 0
    return f


def update_stresses_maxwell(xyz, conn, E, nu, mu, u_n, u_next, dt, stress_n):
    """update_stresses_maxwell (mechanics/stress_update.rs:39-143): [E, 6]."""
    xyz, conn = _f64(xyz), _i64(conn)
    out = np.empty((conn.shape[0], 6))
    assert lib().orc_update_stresses_maxwell(xyz.shape[0], _d(xyz), conn.shape[0], _i(conn), float(E), float(nu),
                                             float(mu), _d(_f64(u_n)), _d(_f64(u_next)), float(dt),
                                             _d(_f64(stress_n)), _d(out)) == 0
    return out


# ------------------------------------------------------------------- problem setups
def thermal_bc(xyz, lz, t_bottom=1280.0, t_top=0.0):
    """Dirichlet set of thermal_1d_improved_mesh.rs:46-52 (|z|<1 -> bottom, |z-lz|<1 -> top)."""
    z = xyz[:, 2]
    bottom = np.abs(z) < 1.0
    top = (~bottom) & (np.abs(z - lz) < 1.0)
    mask = (bottom | top).astype(np.uint8)
    vals = np.where(bottom, t_bottom, np.where(top, t_top, 0.0))
    return mask, vals


# ------------------------------------------------------------------- VTU output
def format_f64(v) -> str:
    """Rust's `{}` for one f64 (core::fmt Display), see vtu.cpp."""
    buf = C.create_string_buffer(400)
    n = lib().orc_format_f64(float(v), buf, 400)
    assert n >= 0
    return buf.raw[:n].decode()


def _field_arrays(fields):
    n = len(fields)
    names = (C.c_char_p * max(n, 1))(*[f[0].encode() for f in fields])
    arrs = [_f64(np.asarray(f[1]).reshape(-1)) for f in fields]
    ptrs = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in arrs])
    comps = np.array([f[2] if len(f) > 2 else 1 for f in fields] or [1], np.int32)
    counts = np.array([a.size // int(c) for a, c in zip(arrs, comps)] or [0], np.int64)
    return n, names, ptrs, counts, comps, arrs


def write_vtu(xyz, conn, point_fields=(), cell_fields=(), fmt="xml") -> bytes:
    """VtkWriter::write_vtu (mesh/vtk_writer.rs:104-265) as bytes; fmt "legacy" gives
    VtkWriter::write (:13-101), "nodal" write_nodal_vtu (:531-789). Fields are
    (name, data, components) with components 1 (scalar) or 3 (vector, [n][3])."""
    fn = {"xml": "orc_write_vtu", "legacy": "orc_write_vtk", "nodal": "orc_write_vtu_nodal"}[fmt]
    xyz = _f64(xyz)
    conn = _i64(conn)
    np_, pn, pp, pc, pk, keep_p = _field_arrays(list(point_fields))
    nc, cn, cp, cc, ck, keep_c = _field_arrays(list(cell_fields))
    L = lib()
    args = (xyz.shape[0], _d(xyz), conn.shape[0], _i(conn), np_, pn, pp, _i(pc), pk.ctypes.data, nc, cn, cp,
            _i(cc), ck.ctypes.data)
    f = getattr(L, fn)
    size = f(*args, None, 0)
    out = C.create_string_buffer(int(size))
    f(*args, out, size)
    return out.raw[:size]
