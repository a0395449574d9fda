"""ctypes binding of libgeofem.so (the C ABI declared in include/geo_fem.h).

The library is built in-tree (``geo_simulator_b200/libgeofem.so``) by
``__graft_entry__.build()`` / ``make -C geo_simulator_b200/csrc``. There is no
CPU fallback: importing works without a GPU, but every compute call raises
``GeoError`` when the library or a B200 is missing.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# GEO_LIBRARY may name another build of the same library (same ABI), e.g. one
# compiled with different launch bounds, to compare builds in one environment.
LIB_PATH = os.environ.get("GEO_LIBRARY") or os.path.join(_HERE, "libgeofem.so")

GEO_OK = 0
GEO_ERR_INVALID_ARG = 1
GEO_VTK_LEGACY, GEO_VTK_XML, GEO_VTK_XML_NODAL = 0, 1, 2
GEO_ERR_SINGULAR_JACOBIAN = 2
GEO_NOT_CONVERGED = 3
GEO_ERR_BREAKDOWN = 4
GEO_ERR_TIMEOUT = 5
GEO_ERR_CUDA = 6
GEO_ERR_UNSUPPORTED = 7
GEO_ERR_NO_DEVICE = 8
GEO_ERR_OUT_OF_MEMORY = 9
GEO_ERR_SINGULAR_MATRIX = 10

PRECISION_FP64 = 0
PRECISION_MIXED = 1

STATUS_NAMES = {
    0: "GEO_OK", 1: "GEO_ERR_INVALID_ARG", 2: "GEO_ERR_SINGULAR_JACOBIAN", 3: "GEO_NOT_CONVERGED",
    4: "GEO_ERR_BREAKDOWN", 5: "GEO_ERR_TIMEOUT", 6: "GEO_ERR_CUDA", 7: "GEO_ERR_UNSUPPORTED",
    8: "GEO_ERR_NO_DEVICE", 9: "GEO_ERR_OUT_OF_MEMORY", 10: "GEO_ERR_SINGULAR_MATRIX",
}


class GeoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class CgOpts(C.Structure):
    _fields_ = [("max_iterations", C.c_int64), ("tolerance", C.c_double), ("abs_tolerance", C.c_double),
                ("use_preconditioner", C.c_int32), ("precision", C.c_int32),
                ("reliable_delta", C.c_double), ("timeout_seconds", C.c_double)]


class SolverStatsC(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("residual_norm", C.c_double),
                ("relative_residual", C.c_double), ("converged", C.c_int32), ("solve_time", C.c_double),
                ("status", C.c_int32), ("fp64_residual_updates", C.c_int64), ("b_norm", C.c_double),
                ("kernel_time", C.c_double), ("kernel_launches", C.c_int64)]


_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_I64 = C.c_int64
_I32 = C.c_int32
_D = C.c_double
_DP = C.c_void_p  # numeric arrays are passed as raw addresses (host or device)

_SIGS = {
    "geo_device_count": [C.POINTER(C.c_int)],
    "geo_ctx_create": [C.c_int, _PP],
    "geo_ctx_destroy": [_P],
    "geo_sm_count": [_P, C.POINTER(C.c_int)],
    "geo_ctx_stream": [_P, _PP],
    "geo_generate_cube_size": [_I64, _I64, _I64, C.POINTER(_I64), C.POINTER(_I64)],
    "geo_generate_cube": [_I64, _I64, _I64, _D, _D, _D, _DP, _DP],
    "geo_mesh_create": [_P, _I64, _DP, _I64, _DP, _PP],
    "geo_mesh_destroy": [_P],
    "geo_mesh_generate_cube": [_P, _I64, _I64, _I64, _D, _D, _D, _PP],
    "geo_mesh_size": [_P, C.POINTER(_I64), C.POINTER(_I64)],
    "geo_mesh_download": [_P, _DP, _DP],
    "geo_vtu_render": [_P, _P, _P, _I32, _P, _I32, _DP, _I64, C.POINTER(_I64)],
    "geo_write_vtu": [_P, _P, _P, _I32, _P, _I32, C.c_char_p, C.POINTER(_I64)],
    "geo_vtk_render": [_P, _P, _I32, _P, _I32, _P, _I32, _DP, _I64, C.POINTER(_I64)],
    "geo_write_vtk": [_P, _P, _I32, _P, _I32, _P, _I32, C.c_char_p, C.POINTER(_I64)],
    "geo_dofs_create": [_P, _I64, _I32, _DP, _DP, _PP],
    "geo_dofs_num_dirichlet": [_P, C.POINTER(_I64)],
    "geo_dofs_destroy": [_P],
    "geo_element_thermal_stiffness": [_P, _P, _DP, _D, _DP],
    "geo_element_thermal_mass": [_P, _P, _D, _D, _DP],
    "geo_element_thermal_load": [_P, _P, _D, _DP],
    "geo_element_elasticity_stiffness": [_P, _P, _DP, _D, _D, _DP],
    "geo_element_gravity_load": [_P, _P, _D, _DP, _DP],
    "geo_assemble_thermal_stiffness": [_P, _P, _P, _DP, _D, _PP],
    "geo_assemble_thermal_load": [_P, _P, _P, _D, _DP],
    "geo_apply_dirichlet_bcs": [_P, _P, _DP, _P, _PP, _DP],
    "geo_assemble_elasticity_stiffness": [_P, _P, _P, _DP, _D, _D, _PP],
    "geo_assemble_gravity_load": [_P, _P, _P, _D, _DP, _DP],
    "geo_csr_create": [_P, _I64, _I64, _I64, _DP, _DP, _DP, _PP],
    "geo_csr_info": [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I64)],
    "geo_csr_copy": [_P, _DP, _DP, _DP],
    "geo_csr_device_ptrs": [_P, _PP, _PP, _PP],
    "geo_csr_apply": [_P, _P, _DP, _DP],
    "geo_csr_destroy": [_P],
    "geo_cg_solve": [_P, _P, _DP, C.POINTER(CgOpts), _DP, C.POINTER(SolverStatsC)],
    "geo_bicgstab_solve": [_P, _P, _DP, C.POINTER(CgOpts), _DP, C.POINTER(SolverStatsC)],
    "geo_gmres_solve": [_P, _P, _DP, C.POINTER(CgOpts), _I32, _DP, C.POINTER(SolverStatsC)],
    "geo_direct_solve": [_P, _P, _DP, _DP, C.POINTER(SolverStatsC)],
    "geo_release_cached_memory": [],
    "geo_device_memory_stats": [C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I64)],
    "geo_thermal_operator_create": [_P, _P, _P, _DP, _D, _PP],
    "geo_elasticity_operator_create": [_P, _P, _P, _DP, _D, _D, _PP],
    "geo_op_set_coefficients": [_P, _DP, _D],
    "geo_op_info": [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_D)],
    "geo_op_apply": [_P, _DP, _DP, _I32],
    "geo_op_lift_rhs": [_P, _DP, _DP],
    "geo_op_diagonal": [_P, _DP],
    "geo_face_flux": [_P, _P, C.c_int64, _DP, _DP, _D, _DP],
    "geo_face_area": [_P, _P, C.c_int64, _DP, _DP],
    "geo_find_boundary_faces": [_P, _P, _DP, C.c_int64, _DP, C.POINTER(C.c_int64)],
    "geo_apply_neumann_bcs": [_P, _P, C.c_int64, _DP, _DP, _D, C.c_int64, _DP],
    "geo_maxwell_history_force": [_P, _P, _DP, _DP],
    "geo_assemble_maxwell_viscoelastic": [_P, _P, _P, _D, _D, _D, _D, _DP, C.POINTER(C.c_void_p), _DP],
    "geo_update_stresses_maxwell": [_P, _P, _D, _D, _D, _DP, _DP, _D, _DP, _DP],
    "geo_cg_solve_noalloc": [_P, _P, _DP, C.POINTER(CgOpts), _DP, C.POINTER(SolverStatsC)],
    "geo_cg_solve_matfree": [_P, _DP, C.POINTER(CgOpts), _DP, C.POINTER(SolverStatsC)],
    "geo_op_element_gradient": [_P, _DP, _DP, _DP],
    "geo_forward": [_P, _DP, C.POINTER(CgOpts), _DP, C.POINTER(SolverStatsC)],
    "geo_vjp": [_P, _DP, _DP, _DP, C.POINTER(CgOpts), _DP, C.POINTER(SolverStatsC)],
    "geo_op_time_pcg_kernels": [_P, _DP, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "geo_op_destroy": [_P],
    "geo_debug_barrier_timeout": [_P, _D],
}

_lib = None


def exported_symbols():
    """Names of every entry point the header declares (for the export test)."""
    return sorted(list(_SIGS) + ["geo_last_error", "geo_version", "geo_cg_opts_default"])


def lib():
    """Load libgeofem.so (raises GeoError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GeoError(GEO_ERR_UNSUPPORTED,
                           f"{LIB_PATH} is missing: run __graft_entry__.build() (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.geo_last_error.argtypes = [_P]
        L.geo_last_error.restype = C.c_char_p
        L.geo_version.argtypes = []
        L.geo_version.restype = C.c_char_p
        L.geo_cg_opts_default.argtypes = [C.POINTER(CgOpts)]
        L.geo_cg_opts_default.restype = None
        _lib = L
    return _lib


def check(code: int, ctx=None, allow=()):
    if code == GEO_OK or code in allow:
        return code
    msg = lib().geo_last_error(ctx).decode(errors="replace") if ctx is not None else \
        lib().geo_last_error(None).decode(errors="replace")
    raise GeoError(code, msg)


def default_opts() -> CgOpts:
    o = CgOpts()
    lib().geo_cg_opts_default(C.byref(o))
    return o
