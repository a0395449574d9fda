"""Host-side mirror of the reference's Tet10 hot-path API over the C ABI.

Names, argument meaning and error behaviour follow msahamed/geo_simulator:

* ``ImprovedMeshGenerator.generate_cube``   -- src/mesh_generator_improved.rs:19-169
* ``Mesh``                                  -- src/mesh/geometry.rs:41-71
* ``DofManager``                            -- src/fem/dof.rs:8-180
* ``ElementMatrix`` / ``ElasticityElement`` / ``BodyForce`` -- src/fem/element.rs,
  src/mechanics/{element,body_force}.rs (batched over every element of a mesh)
* ``Assembler``                             -- src/fem/assembly.rs:22-239, 389-437, 906-937
* ``ConjugateGradient`` / ``SolverStats``   -- src/linalg/iterative.rs:7-147, solver.rs:5-32
* ``IsotropicElasticity``                   -- src/mechanics/constitutive.rs:15-102

Every numeric call runs on the GPU through libgeofem.so; there is no CPU
fallback. Arrays may be numpy (host) or torch CUDA tensors (device).
Reference panics (singular Jacobian, wrong DOFs per node) raise ``GeoError``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from ._native import GeoError

__all__ = [
    "Context", "Mesh", "ImprovedMeshGenerator", "DofManager", "IsotropicElasticity", "CsrMatrix",
    "ElementMatrix", "ElasticityElement", "BodyForce", "Assembler", "SolverStats", "ConjugateGradient",
    "ThermalOperator", "ElasticityOperator", "GeoError", "BoundaryFace", "NeumannBC", "BoundaryConditions",
    "Tet10Face", "MaxwellViscoelasticity", "StressHistory", "BackwardEuler", "TimeStepStats",
    "update_stresses_maxwell",
]


# --------------------------------------------------------------------------- plumbing
def _ptr(a):
    """Raw address of a numpy array or torch tensor (must be contiguous)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


def _f64(a):
    if hasattr(a, "data_ptr") and not isinstance(a, np.ndarray):
        import torch
        if a.dtype != torch.float64:
            raise TypeError("expected a float64 tensor")
        return a.contiguous()
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One CUDA context/stream of libgeofem (geo_ctx)."""

    _default: dict[int, "Context"] = {}

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        N.check(N.lib().geo_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = Context(device)
        return cls._default[device]

    def check(self, code, allow=()):
        return N.check(code, self.h, allow)

    def stream_handle(self) -> int:
        """cudaStream_t of this context (for torch.cuda.ExternalStream)."""
        v = C.c_void_p()
        self.check(N.lib().geo_ctx_stream(self.h, C.byref(v)))
        return v.value or 0

    def sm_count(self) -> int:
        v = C.c_int()
        self.check(N.lib().geo_sm_count(self.h, C.byref(v)))
        return v.value

    def __del__(self):
        try:
            if getattr(self, "h", None):
                N.lib().geo_ctx_destroy(self.h)
        except Exception:
            pass


def _ctx(ctx):
    return ctx if ctx is not None else Context.default()


# --------------------------------------------------------------------------- mesh
class Mesh:
    """Tet10 mesh: ``nodes`` float64 [N, 3], ``elements`` int32 [E, 10]."""

    def __init__(self, nodes, elements):
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64).reshape(-1, 3)
        el = np.asarray(elements)
        if el.size and (el.min() < 0 or el.max() >= self.nodes.shape[0]):
            raise GeoError(N.GEO_ERR_INVALID_ARG, "element references a node id out of range")
        self.elements = np.ascontiguousarray(el, dtype=np.int32).reshape(-1, 10)
        self._handles = {}
        self.stress_history = None  # StressHistory for viscoelasticity (mesh/geometry.rs)
        self.field_data, self.cell_data = FieldData(), FieldData()  # mesh/geometry.rs:44-45

    def num_nodes(self) -> int:
        return int(self.nodes.shape[0])

    def num_elements(self) -> int:
        return int(self.elements.shape[0])

    def handle(self, ctx=None):
        ctx = _ctx(ctx)
        key = id(ctx)
        if key not in self._handles:
            h = C.c_void_p()
            ctx.check(N.lib().geo_mesh_create(ctx.h, self.num_nodes(), _ptr(self.nodes), self.num_elements(),
                                              _ptr(self.elements), C.byref(h)))
            self._handles[key] = (ctx, h)
        return self._handles[key][1]

    def __del__(self):
        for ctx, h in getattr(self, "_handles", {}).values():
            try:
                N.lib().geo_mesh_destroy(h)
            except Exception:
                pass


class ImprovedMeshGenerator:
    """mesh_generator_improved.rs:8-170 (6 tets per hex, shared edge midpoints)."""

    @staticmethod
    def generate_cube(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float) -> Mesh:
        L = N.lib()
        n_nodes, n_elem = C.c_int64(), C.c_int64()
        N.check(L.geo_generate_cube_size(nx, ny, nz, C.byref(n_nodes), C.byref(n_elem)))
        xyz = np.empty((n_nodes.value, 3), np.float64)
        conn = np.empty((n_elem.value, 10), np.int32)
        N.check(L.geo_generate_cube(nx, ny, nz, float(lx), float(ly), float(lz), _ptr(xyz), _ptr(conn)))
        m = Mesh.__new__(Mesh)
        m.nodes, m.elements, m._handles, m.stress_history = xyz, conn, {}, None
        m.field_data, m.cell_data = FieldData(), FieldData()
        return m

    @staticmethod
    def generate_cube_device(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float, ctx=None) -> "DeviceMesh":
        """``generate_cube`` run on the GPU: the mesh is built in device memory
        (same numbering, coordinates and connectivity, bit for bit) and the host
        arrays are only downloaded when ``nodes`` / ``elements`` are read."""
        ctx = _ctx(ctx)
        h = C.c_void_p()
        ctx.check(N.lib().geo_mesh_generate_cube(ctx.h, nx, ny, nz, float(lx), float(ly), float(lz), C.byref(h)))
        return DeviceMesh(ctx, h)


class DeviceMesh(Mesh):
    """A Mesh whose primary copy lives on the device (``geo_mesh``); ``nodes`` and
    ``elements`` are the reference's host arrays, copied out on first access."""

    def __init__(self, ctx, h):
        n_nodes, n_elem = C.c_int64(), C.c_int64()
        ctx.check(N.lib().geo_mesh_size(h, C.byref(n_nodes), C.byref(n_elem)))
        self._n_nodes, self._n_elem = int(n_nodes.value), int(n_elem.value)
        self._handles = {id(ctx): (ctx, h)}
        self._ctx = ctx
        self._nodes = self._elements = None
        self.stress_history = None
        self.field_data, self.cell_data = FieldData(), FieldData()

    def num_nodes(self) -> int:
        return self._n_nodes

    def num_elements(self) -> int:
        return self._n_elem

    def _download(self, nodes: bool):
        h = self._handles[id(self._ctx)][1]
        if nodes:
            xyz = np.empty((self._n_nodes, 3), np.float64)
            self._ctx.check(N.lib().geo_mesh_download(h, _ptr(xyz), None))
            self._nodes = xyz
        else:
            conn = np.empty((self._n_elem, 10), np.int32)
            self._ctx.check(N.lib().geo_mesh_download(h, None, _ptr(conn)))
            self._elements = conn

    @property
    def nodes(self):
        if self._nodes is None:
            self._download(True)
        return self._nodes

    @nodes.setter
    def nodes(self, value):
        self._nodes = value

    @property
    def elements(self):
        if self._elements is None:
            self._download(False)
        return self._elements

    @elements.setter
    def elements(self, value):
        self._elements = value


# --------------------------------------------------------------------------- fields and VTU output
class ScalarField:
    """mesh/fields.rs:4-26: a named value per node (or per cell)."""

    def __init__(self, name: str, data):
        self.name, self.data = str(name), data

    new = classmethod(lambda cls, name, data: cls(name, data))

    def len(self) -> int:
        return int(np.asarray(self.data).size) if not hasattr(self.data, "numel") else int(self.data.numel())


class VectorField:
    """mesh/fields.rs:28-76: a named 3-vector per node (or per cell), stored [n][3]."""

    def __init__(self, name: str, data):
        self.name, self.data = str(name), data

    new = classmethod(lambda cls, name, data: cls(name, data))

    @classmethod
    def from_dof_vector(cls, name: str, dof_vector):
        """fields.rs:54-66: interleaved [x0 y0 z0 x1 ...]; panics unless 3 | len."""
        n = dof_vector.numel() if hasattr(dof_vector, "numel") else np.asarray(dof_vector).size
        if n % 3:
            raise GeoError(N.GEO_ERR_INVALID_ARG, "DOF vector must have 3*n entries for vector field")
        return cls(name, dof_vector)

    def len(self) -> int:
        n = self.data.numel() if hasattr(self.data, "numel") else np.asarray(self.data).size
        return int(n) // 3


class FieldData:
    """mesh/fields.rs:78-137. The reference keys HashMaps (unspecified order);
    these dicts keep insertion order, which VtkWriter writes."""

    def __init__(self):
        self.scalar_fields: dict[str, ScalarField] = {}
        self.vector_fields: dict[str, VectorField] = {}

    new = classmethod(lambda cls: cls())

    def add_field(self, field: ScalarField):
        self.scalar_fields[field.name] = field

    def add_vector_field(self, field: VectorField):
        self.vector_fields[field.name] = field

    def get_field(self, name):
        return self.scalar_fields.get(name)

    def get_vector_field(self, name):
        return self.vector_fields.get(name)

    def field_names(self):
        return list(self.scalar_fields)

    def vector_field_names(self):
        return list(self.vector_fields)

    def num_fields(self) -> int:
        return len(self.scalar_fields)

    def num_vector_fields(self) -> int:
        return len(self.vector_fields)

    def is_empty(self) -> bool:
        return not self.scalar_fields and not self.vector_fields


class _VtuField(C.Structure):
    _fields_ = [("name", C.c_char_p), ("data", C.c_void_p), ("count", C.c_int64), ("components", C.c_int32)]


def _vtu_fields(fd: FieldData):
    keep, out = [], []
    for f, comps in [(f, 1) for f in fd.scalar_fields.values()] + [(f, 3) for f in fd.vector_fields.values()]:
        d = f.data
        if hasattr(d, "is_cuda"):
            d = d.detach().to(dtype=__import__("torch").float64).contiguous()
            n = d.numel()
        else:
            d = np.ascontiguousarray(d, dtype=np.float64).reshape(-1)
            n = d.size
        keep.append(d)
        out.append(_VtuField(f.name.encode(), _ptr(d), n // comps, comps))
    arr = (_VtuField * max(1, len(out)))(*out)
    return arr, len(out), keep


class VtkWriter:
    """mesh/vtk_writer.rs:7-789: the text is rendered on the GPU, byte for byte as
    the reference's writers (Rust ``{}`` for every number)."""

    @staticmethod
    def _out(mesh, fmt, filename, out, ctx):
        ctx = _ctx(ctx)
        pf, npf, k1 = _vtu_fields(mesh.field_data)
        cf, ncf, k2 = _vtu_fields(mesh.cell_data)
        L = N.lib()
        size = C.c_int64()
        h = mesh.handle(ctx)
        if filename is not None:
            ctx.check(L.geo_write_vtk(ctx.h, h, fmt, pf, npf, cf, ncf, str(filename).encode(), C.byref(size)))
            return int(size.value)
        if out is not None:
            cap = out.numel() if hasattr(out, "numel") else out.size
            ctx.check(L.geo_vtk_render(ctx.h, h, fmt, pf, npf, cf, ncf, _ptr(out), cap, C.byref(size)))
            return int(size.value)
        ctx.check(L.geo_vtk_render(ctx.h, h, fmt, pf, npf, cf, ncf, None, 0, C.byref(size)))
        buf = np.empty(int(size.value), np.uint8)
        ctx.check(L.geo_vtk_render(ctx.h, h, fmt, pf, npf, cf, ncf, _ptr(buf), buf.size, C.byref(size)))
        return buf.tobytes()

    @staticmethod
    def write(mesh: Mesh, filename: str, ctx=None) -> int:
        """VtkWriter::write (vtk_writer.rs:13-101): legacy ASCII .vtk; returns the bytes written."""
        return VtkWriter._out(mesh, N.GEO_VTK_LEGACY, filename, None, ctx)

    @staticmethod
    def write_vtu(mesh: Mesh, filename: str, ctx=None) -> int:
        """VtkWriter::write_vtu (vtk_writer.rs:104-265); returns the bytes written."""
        return VtkWriter._out(mesh, N.GEO_VTK_XML, filename, None, ctx)

    @staticmethod
    def write_nodal_vtu(mesh: Mesh, tracers, filename: str, ctx=None) -> int:
        """VtkWriter::write_nodal_vtu (vtk_writer.rs:531-789); the tracers are unused, as
        in the reference. Returns the bytes written."""
        return VtkWriter._out(mesh, N.GEO_VTK_XML_NODAL, filename, None, ctx)

    @staticmethod
    def render_vtu(mesh: Mesh, out=None, ctx=None, fmt=None):
        """The text of write_vtu (or of ``fmt``: GEO_VTK_LEGACY / _XML / _XML_NODAL) as
        bytes (out None), or into ``out`` (a uint8 numpy array or CUDA tensor large
        enough); returns the bytes or the size."""
        return VtkWriter._out(mesh, N.GEO_VTK_XML if fmt is None else fmt, None, out, ctx)


class VtkFormat:
    """vtk_writer.rs:791-845."""
    Legacy, Xml, XmlNodal, XmlMultiBlock = "Legacy", "Xml", "XmlNodal", "XmlMultiBlock"
    _EXT = {"Legacy": ".vtk", "Xml": ".vtu", "XmlNodal": ".vtu", "XmlMultiBlock": ".vtm"}

    @staticmethod
    def extension(fmt) -> str:
        return VtkFormat._EXT[fmt]

    @staticmethod
    def from_filename(filename: str):
        if filename.endswith(".vtk"):
            return VtkFormat.Legacy
        if filename.endswith(".vtu"):
            return VtkFormat.XmlNodal  # the reference's default for .vtu
        if filename.endswith(".vtm"):
            return VtkFormat.XmlMultiBlock
        return None


class VtkOutputBuilder:
    """vtk_writer.rs:847-985 (default format XmlNodal; with_fields is stored but, as in
    the reference, not applied). The tracer multi-block format has no GPU writer here."""

    def __init__(self, mesh: Mesh):
        self.mesh, self.tracers, self.format, self.fields = mesh, None, VtkFormat.XmlNodal, None

    new = classmethod(lambda cls, mesh: cls(mesh))

    def with_tracers(self, tracers):
        self.tracers = tracers
        return self

    def with_format(self, fmt):
        self.format = fmt
        return self

    def with_fields(self, fields):
        self.fields = list(fields)
        return self

    def auto_format(self, filename: str):
        fmt = VtkFormat.from_filename(filename)
        if fmt is not None:
            self.format = fmt
        return self

    def write(self, filename: str, ctx=None) -> int:
        if self.format == VtkFormat.Legacy:
            return VtkWriter.write(self.mesh, filename, ctx)
        if self.format == VtkFormat.Xml:
            return VtkWriter.write_vtu(self.mesh, filename, ctx)
        if self.format == VtkFormat.XmlNodal:
            return VtkWriter.write_nodal_vtu(self.mesh, self.tracers, filename, ctx)
        raise GeoError(N.GEO_ERR_UNSUPPORTED, "the multi-block tracer format (write_combined_vtu) is not supported")

    def recommended_filename(self, base: str) -> str:
        return base + VtkFormat.extension(self.format)


def quick_write_vtu(mesh: Mesh, filename: str, ctx=None) -> int:
    """vtk_writer.rs:986-988: the builder's default (nodal) format."""
    return VtkOutputBuilder(mesh).write(filename, ctx)


# --------------------------------------------------------------------------- DOFs
class DofManager:
    """dof.rs:8-180 for a fixed number of DOFs per node (``new``, :37-50)."""

    def __init__(self, num_nodes: int, dofs_per_node: int):
        self._num_nodes = int(num_nodes)
        self._dpn = int(dofs_per_node)
        self._mask = np.zeros(self._num_nodes * self._dpn, np.uint8)
        self._values = np.zeros(self._num_nodes * self._dpn, np.float64)
        self._handles = {}

    # dof.rs:87-106
    def global_dof(self, node_id: int, local_dof: int) -> int:
        if local_dof >= self._dpn:
            raise GeoError(N.GEO_ERR_INVALID_ARG, "Node has no pressure DOF")
        return node_id * self._dpn + local_dof

    velocity_dof = global_dof

    # dof.rs:113-130
    def set_dirichlet(self, dof, value):
        self._mask[dof] = 1
        self._values[dof] = value
        self._handles.clear()

    def set_dirichlet_node(self, node_id, value):
        for c in range(self._dpn):
            self.set_dirichlet(np.asarray(node_id) * self._dpn + c, value)

    def is_dirichlet(self, dof) -> bool:
        return bool(self._mask[dof])

    def get_dirichlet_value(self, dof) -> float:
        return float(self._values[dof])

    def total_dofs(self) -> int:
        return self._num_nodes * self._dpn

    def num_free_dofs(self) -> int:
        return self.total_dofs() - int(self._mask.sum())

    def num_constrained_dofs(self) -> int:
        return int(self._mask.sum())

    def dofs_per_node(self) -> int:
        return self._dpn

    def num_nodes(self) -> int:
        return self._num_nodes

    @property
    def dirichlet_mask(self):
        return self._mask

    @property
    def dirichlet_values(self):
        return self._values

    def handle(self, ctx=None):
        ctx = _ctx(ctx)
        key = id(ctx)
        if key not in self._handles:
            h = C.c_void_p()
            ctx.check(N.lib().geo_dofs_create(ctx.h, self._num_nodes, self._dpn, _ptr(self._mask),
                                              _ptr(self._values), C.byref(h)))
            self._handles[key] = _DofsHandle(h)
        return self._handles[key].h


class _DofsHandle:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        try:
            N.lib().geo_dofs_destroy(self.h)
        except Exception:
            pass


# --------------------------------------------------------------------------- material
@dataclass
class IsotropicElasticity:
    """constitutive.rs:15-41 (E > 0, -1 < nu < 0.5)."""
    youngs_modulus: float
    poisson_ratio: float

    def __post_init__(self):
        if not self.youngs_modulus > 0.0:
            raise GeoError(N.GEO_ERR_INVALID_ARG, "Young's modulus must be positive")
        if not (-1.0 < self.poisson_ratio < 0.5):
            raise GeoError(N.GEO_ERR_INVALID_ARG, "Poisson's ratio must be in (-1, 0.5) for physical stability")

    @staticmethod
    def new(youngs_modulus, poisson_ratio):
        return IsotropicElasticity(youngs_modulus, poisson_ratio)


# --------------------------------------------------------------------------- CSR
class CsrMatrix:
    """Device-resident CSR (the sprs CsMat<f64> the reference returns)."""

    def __init__(self, h, ctx):
        self.h, self.ctx = h, ctx
        r, c, z = C.c_int64(), C.c_int64(), C.c_int64()
        N.check(N.lib().geo_csr_info(h, C.byref(r), C.byref(c), C.byref(z)))
        self._shape = (r.value, c.value)
        self._nnz = z.value

    @classmethod
    def from_arrays(cls, n_rows, n_cols, indptr, indices, data, ctx=None):
        ctx = _ctx(ctx)
        indptr = np.ascontiguousarray(indptr, np.int64)
        indices = np.ascontiguousarray(indices, np.int32)
        data = np.ascontiguousarray(data, np.float64)
        h = C.c_void_p()
        ctx.check(N.lib().geo_csr_create(ctx.h, n_rows, n_cols, indices.size, _ptr(indptr), _ptr(indices),
                                         _ptr(data), C.byref(h)))
        return cls(h, ctx)

    @classmethod
    def from_triplets(cls, n_rows, n_cols, rows, cols, vals, ctx=None):
        """TriMat::add_triplet + to_csr (duplicates summed, explicit zeros kept)."""
        rows, cols = np.asarray(rows, np.int64), np.asarray(cols, np.int64)
        vals = np.asarray(vals, np.float64)
        order = np.lexsort((cols, rows))
        r, c, v = rows[order], cols[order], vals[order]
        key = r * n_cols + c
        uniq, start = np.unique(key, return_index=True)
        data = np.add.reduceat(v, start) if v.size else v
        ur, uc = uniq // n_cols, uniq % n_cols
        indptr = np.zeros(n_rows + 1, np.int64)
        np.add.at(indptr, ur + 1, 1)
        return cls.from_arrays(n_rows, n_cols, np.cumsum(indptr), uc, data, ctx)

    def rows(self):
        return self._shape[0]

    def cols(self):
        return self._shape[1]

    def nnz(self):
        return self._nnz

    @property
    def shape(self):
        return self._shape

    def to_host(self):
        ip = np.empty(self._shape[0] + 1, np.int64)
        ix = np.empty(self._nnz, np.int32)
        d = np.empty(self._nnz, np.float64)
        self.ctx.check(N.lib().geo_csr_copy(self.h, _ptr(ip), _ptr(ix), _ptr(d)))
        return ip, ix, d

    def to_scipy(self):
        import scipy.sparse as sp
        ip, ix, d = self.to_host()
        return sp.csr_matrix((d, ix, ip), shape=self._shape)

    def apply(self, x):
        """LinearOperator::apply (solver.rs:61-73)."""
        x = _f64(x)
        y = np.empty(self._shape[0]) if isinstance(x, np.ndarray) else x.new_empty(self._shape[0])
        self.ctx.check(N.lib().geo_csr_apply(self.ctx.h, self.h, _ptr(x), _ptr(y)))
        return y

    def __del__(self):
        try:
            N.lib().geo_csr_destroy(self.h)
        except Exception:
            pass


# --------------------------------------------------------------------------- elements
def _coef_ptr(coef, n_elem):
    if np.isscalar(coef):
        return None, float(coef), None
    a = _f64(coef)
    if a.shape[0] != n_elem:
        raise GeoError(N.GEO_ERR_INVALID_ARG, "per-element coefficient array has the wrong length")
    return _ptr(a), 0.0, a


class ElementMatrix:
    """element.rs:8-140, batched: one matrix per element of ``mesh``."""

    @staticmethod
    def thermal_stiffness(mesh: Mesh, conductivity, ctx=None):
        ctx = _ctx(ctx)
        p, k, keep = _coef_ptr(conductivity, mesh.num_elements())
        out = np.empty((mesh.num_elements(), 10, 10))
        ctx.check(N.lib().geo_element_thermal_stiffness(ctx.h, mesh.handle(ctx), p, k, _ptr(out)))
        return out

    @staticmethod
    def thermal_mass(mesh: Mesh, density, specific_heat, ctx=None):
        ctx = _ctx(ctx)
        out = np.empty((mesh.num_elements(), 10, 10))
        ctx.check(N.lib().geo_element_thermal_mass(ctx.h, mesh.handle(ctx), float(density),
                                                   float(specific_heat), _ptr(out)))
        return out

    @staticmethod
    def thermal_load(mesh: Mesh, source, ctx=None):
        ctx = _ctx(ctx)
        out = np.empty((mesh.num_elements(), 10))
        ctx.check(N.lib().geo_element_thermal_load(ctx.h, mesh.handle(ctx), float(source), _ptr(out)))
        return out


class ElasticityElement:
    """mechanics/element.rs:33-65, batched."""

    @staticmethod
    def stiffness_matrix(mesh: Mesh, material: IsotropicElasticity, youngs_e=None, ctx=None):
        ctx = _ctx(ctx)
        ee = None if youngs_e is None else _f64(youngs_e)
        out = np.empty((mesh.num_elements(), 30, 30))
        ctx.check(N.lib().geo_element_elasticity_stiffness(ctx.h, mesh.handle(ctx), _ptr(ee),
                                                           float(material.youngs_modulus),
                                                           float(material.poisson_ratio), _ptr(out)))
        return out


class BodyForce:
    """mechanics/body_force.rs:49-84, batched."""

    @staticmethod
    def gravity_load(mesh: Mesh, density, gravity, ctx=None):
        ctx = _ctx(ctx)
        g = np.ascontiguousarray(gravity, np.float64)
        out = np.empty((mesh.num_elements(), 30))
        ctx.check(N.lib().geo_element_gravity_load(ctx.h, mesh.handle(ctx), float(density), _ptr(g), _ptr(out)))
        return out


# --------------------------------------------------------------------------- assembly
class Assembler:
    """assembly.rs:7-1021 (the hot-path subset)."""

    @staticmethod
    def assemble_thermal_stiffness_parallel(mesh: Mesh, dof_mgr: DofManager, conductivity, ctx=None):
        ctx = _ctx(ctx)
        p, k, keep = _coef_ptr(conductivity, mesh.num_elements())
        h = C.c_void_p()
        ctx.check(N.lib().geo_assemble_thermal_stiffness(ctx.h, mesh.handle(ctx), dof_mgr.handle(ctx), p, k,
                                                         C.byref(h)))
        return CsrMatrix(h, ctx)

    # the serial variant has the same result (assembly.rs:22-58)
    assemble_thermal_stiffness_serial = assemble_thermal_stiffness_parallel

    @staticmethod
    def assemble_thermal_load(mesh: Mesh, dof_mgr: DofManager, source, ctx=None):
        ctx = _ctx(ctx)
        f = np.empty(dof_mgr.total_dofs())
        ctx.check(N.lib().geo_assemble_thermal_load(ctx.h, mesh.handle(ctx), dof_mgr.handle(ctx), float(source),
                                                    _ptr(f)))
        return f

    @staticmethod
    def apply_dirichlet_bcs(K: CsrMatrix, f, dof_mgr: DofManager, ctx=None):
        ctx = ctx or K.ctx
        f = _f64(f)
        h = C.c_void_p()
        fbc = np.empty(K.rows())
        ctx.check(N.lib().geo_apply_dirichlet_bcs(ctx.h, K.h, _ptr(f), dof_mgr.handle(ctx), C.byref(h), _ptr(fbc)))
        return CsrMatrix(h, ctx), fbc

    @staticmethod
    def apply_dirichlet_bcs_only_matrix(K: CsrMatrix, dof_mgr: DofManager, ctx=None):
        return Assembler.apply_dirichlet_bcs(K, np.zeros(K.rows()), dof_mgr, ctx)[0]

    @staticmethod
    def assemble_elasticity_stiffness_parallel(mesh: Mesh, dof_mgr: DofManager, material: IsotropicElasticity,
                                               youngs_e=None, ctx=None):
        ctx = _ctx(ctx)
        ee = None if youngs_e is None else _f64(youngs_e)
        h = C.c_void_p()
        ctx.check(N.lib().geo_assemble_elasticity_stiffness(ctx.h, mesh.handle(ctx), dof_mgr.handle(ctx),
                                                            _ptr(ee), float(material.youngs_modulus),
                                                            float(material.poisson_ratio), C.byref(h)))
        return CsrMatrix(h, ctx)

    assemble_elasticity_stiffness_serial = assemble_elasticity_stiffness_parallel

    @staticmethod
    def find_boundary_faces(mesh: Mesh, condition, ctx=None):
        """assembly.rs:287-309. ``condition`` is a callable on the node coordinates
        (an [N, 3] array, vectorised) returning a boolean per node, or a boolean
        mask itself. Returns [(element_id, local_face_id)] as an int32 [n, 2] array."""
        ctx = _ctx(ctx)
        mask = condition(mesh.nodes) if callable(condition) else condition
        mask = np.ascontiguousarray(np.asarray(mask, bool).astype(np.uint8))
        if mask.shape != (mesh.num_nodes(),):
            raise GeoError(N.GEO_ERR_INVALID_ARG, "condition must give one value per node")
        n = C.c_int64()
        L = N.lib()
        ctx.check(L.geo_find_boundary_faces(ctx.h, mesh.handle(ctx), _ptr(mask), 0, None, C.byref(n)))
        faces = np.empty((n.value, 2), np.int32)
        if n.value:
            ctx.check(L.geo_find_boundary_faces(ctx.h, mesh.handle(ctx), _ptr(mask), n.value, _ptr(faces),
                                                C.byref(n)))
        return faces

    @staticmethod
    def apply_neumann_bcs(mesh: Mesh, f, bcs, ctx=None):
        """assembly.rs:248-274: f[node] += face flux contributions, in place.
        ``bcs`` is a BoundaryConditions or a (faces [n, 2], flux) pair."""
        ctx = _ctx(ctx)
        faces, flux = bcs.arrays() if isinstance(bcs, BoundaryConditions) else bcs
        faces = np.ascontiguousarray(faces, np.int32).reshape(-1, 2)
        fl = np.asarray(flux, np.float64)
        flp = np.ascontiguousarray(np.broadcast_to(fl, (faces.shape[0],))) if fl.ndim > 0 else None
        if not (isinstance(f, np.ndarray) and f.dtype == np.float64 and f.flags["C_CONTIGUOUS"]) and \
                not hasattr(f, "data_ptr"):
            raise TypeError("f must be a contiguous float64 array (updated in place)")
        n_f = f.shape[0] if isinstance(f, np.ndarray) else f.numel()
        ctx.check(N.lib().geo_apply_neumann_bcs(ctx.h, mesh.handle(ctx), faces.shape[0], _ptr(faces), _ptr(flp),
                                                float(fl) if fl.ndim == 0 else 0.0, n_f, _ptr(f)))
        return f

    @staticmethod
    def maxwell_history_force(mesh: Mesh, stress_history, ctx=None):
        """f_history of assemble_maxwell_viscoelastic_parallel (assembly.rs:959-1020)."""
        ctx = _ctx(ctx)
        st = stress_history.stress if isinstance(stress_history, StressHistory) else stress_history
        st = np.ascontiguousarray(st, np.float64)
        f = np.empty(3 * mesh.num_nodes())
        ctx.check(N.lib().geo_maxwell_history_force(ctx.h, mesh.handle(ctx), _ptr(st), _ptr(f)))
        return f

    @staticmethod
    def assemble_maxwell_viscoelastic_parallel(mesh: Mesh, dof_mgr: DofManager, material, dt, ctx=None):
        """assembly.rs:959-1020: (elastic K, f_history) from mesh.stress_history."""
        ctx = _ctx(ctx)
        if mesh.stress_history is None:
            raise GeoError(N.GEO_ERR_INVALID_ARG, "Mesh must have stress_history for viscoelasticity")
        st = np.ascontiguousarray(mesh.stress_history.stress, np.float64)
        h = C.c_void_p()
        f = np.empty(dof_mgr.total_dofs())
        ctx.check(N.lib().geo_assemble_maxwell_viscoelastic(ctx.h, mesh.handle(ctx), dof_mgr.handle(ctx),
                                                            material.youngs_modulus, material.poisson_ratio,
                                                            material.viscosity, float(dt), _ptr(st), C.byref(h),
                                                            _ptr(f)))
        return CsrMatrix(h, ctx), f

    @staticmethod
    def assemble_gravity_load(mesh: Mesh, dof_mgr: DofManager, density, gravity, ctx=None):
        ctx = _ctx(ctx)
        g = np.ascontiguousarray(gravity, np.float64)
        f = np.empty(dof_mgr.total_dofs())
        ctx.check(N.lib().geo_assemble_gravity_load(ctx.h, mesh.handle(ctx), dof_mgr.handle(ctx), float(density),
                                                    _ptr(g), _ptr(f)))
        return f


# --------------------------------------------------------------------------- Neumann boundary
@dataclass(frozen=True)
class BoundaryFace:
    """boundary.rs:9-15: (element, local face); local face f is opposite vertex f."""
    element_id: int
    local_face_id: int


@dataclass
class NeumannBC:
    """boundary.rs:18-23: prescribed flux on a face."""
    flux: float


class BoundaryConditions:
    """boundary.rs:26-59: the Neumann faces and their fluxes (insertion order kept)."""

    def __init__(self):
        self._neumann = {}

    @staticmethod
    def new():
        return BoundaryConditions()

    def add_neumann(self, face: BoundaryFace, flux: float):
        self._neumann[face] = NeumannBC(float(flux))

    def get_neumann(self, face: BoundaryFace):
        return self._neumann.get(face)

    def neumann_faces(self):
        return list(self._neumann.items())

    def num_neumann_bcs(self) -> int:
        return len(self._neumann)

    def arrays(self):
        """(faces int32 [n, 2], flux float64 [n]) in insertion order."""
        items = self.neumann_faces()
        faces = np.array([[f.element_id, f.local_face_id] for f, _ in items], np.int32).reshape(-1, 2)
        flux = np.array([bc.flux for _, bc in items], np.float64)
        return faces, flux


class Tet10Face:
    """boundary.rs:66-267: a 6-node face of a Tet10 (3 vertices then 3 midpoints)."""

    # local element node of each face node, boundary.rs:91-127
    FACE_NODES = np.array([[1, 2, 3, 5, 9, 8], [0, 2, 3, 6, 9, 7], [0, 1, 3, 4, 8, 7], [0, 1, 2, 4, 5, 6]],
                          np.int32)

    def __init__(self, nodes):
        self.nodes = np.asarray(nodes, np.int64)

    @staticmethod
    def from_element_face(element_nodes, local_face: int) -> "Tet10Face":
        if not 0 <= int(local_face) <= 3:
            raise GeoError(N.GEO_ERR_INVALID_ARG, f"Invalid face index for tet10: {local_face}")
        return Tet10Face(np.asarray(element_nodes)[Tet10Face.FACE_NODES[int(local_face)]])

    @staticmethod
    def integrate_flux_faces(mesh: Mesh, faces, flux, ctx=None):
        """integrate_flux for many (element, local face) pairs on the GPU: [n, 6]."""
        ctx = _ctx(ctx)
        faces = np.ascontiguousarray(faces, np.int32).reshape(-1, 2)
        fl = np.asarray(flux, np.float64)
        per_face = fl.ndim > 0
        flp = np.ascontiguousarray(np.broadcast_to(fl, (faces.shape[0],))) if per_face else None
        out = np.empty((faces.shape[0], 6))
        ctx.check(N.lib().geo_face_flux(ctx.h, mesh.handle(ctx), faces.shape[0], _ptr(faces), _ptr(flp),
                                        float(fl) if not per_face else 0.0, _ptr(out)))
        return out

    @staticmethod
    def area_faces(mesh: Mesh, faces, ctx=None):
        """area for many faces on the GPU."""
        ctx = _ctx(ctx)
        faces = np.ascontiguousarray(faces, np.int32).reshape(-1, 2)
        out = np.empty(faces.shape[0])
        ctx.check(N.lib().geo_face_area(ctx.h, mesh.handle(ctx), faces.shape[0], _ptr(faces), _ptr(out)))
        return out


# --------------------------------------------------------------------------- Maxwell viscoelasticity
@dataclass
class MaxwellViscoelasticity:
    """mechanics/constitutive.rs:286-395: E (Pa), nu, viscosity mu (Pa s)."""
    youngs_modulus: float
    poisson_ratio: float
    viscosity: float

    def __post_init__(self):
        if not self.youngs_modulus > 0:
            raise GeoError(N.GEO_ERR_INVALID_ARG, f"Young's modulus must be positive, got {self.youngs_modulus}")
        if not -1.0 < self.poisson_ratio < 0.5:
            raise GeoError(N.GEO_ERR_INVALID_ARG, f"Poisson's ratio must be in (-1, 0.5), got {self.poisson_ratio}")
        if not self.viscosity > 0:
            raise GeoError(N.GEO_ERR_INVALID_ARG, f"Viscosity must be positive, got {self.viscosity}")

    @staticmethod
    def new(youngs_modulus, poisson_ratio, viscosity):
        return MaxwellViscoelasticity(float(youngs_modulus), float(poisson_ratio), float(viscosity))

    def shear_modulus(self) -> float:
        return self.youngs_modulus / (2.0 * (1.0 + self.poisson_ratio))

    def relaxation_time(self) -> float:
        return self.viscosity / self.shear_modulus()

    def elastic_matrix(self):
        """IsotropicElasticity::constitutive_matrix (Voigt, engineering shear)."""
        E, nu = self.youngs_modulus, self.poisson_ratio
        f = E / ((1.0 + nu) * (1.0 - 2.0 * nu))
        D = np.zeros((6, 6))
        D[:3, :3] = nu
        np.fill_diagonal(D[:3, :3], 1.0 - nu)
        D[3, 3] = D[4, 4] = D[5, 5] = (1.0 - 2.0 * nu) / 2.0
        return f * D

    def effective_constitutive_matrix(self, dt):
        """D_elastic / (1 + dt / tau_M)."""
        return self.elastic_matrix() / (1.0 + dt / self.relaxation_time())


class StressHistory:
    """mesh/state.rs:12-75: Voigt stress [xx yy zz xy yz zx] per element."""

    def __init__(self, n_elements: int):
        self.stress = np.zeros((int(n_elements), 6))

    @staticmethod
    def new(n_elements):
        return StressHistory(n_elements)

    def get(self, elem_id):
        return self.stress[elem_id]

    def set(self, elem_id, stress):
        self.stress[elem_id] = stress

    def update_all(self, new_stresses):
        self.stress = np.ascontiguousarray(new_stresses, np.float64).reshape(-1, 6)

    def num_elements(self):
        return self.stress.shape[0]


def update_stresses_maxwell(mesh: Mesh, dof_mgr: DofManager, material: MaxwellViscoelasticity, u_n, u_next, dt,
                            ctx=None):
    """mechanics/stress_update.rs:39-143: new [E, 6] stresses from mesh.stress_history."""
    ctx = _ctx(ctx)
    if mesh.stress_history is None:
        raise GeoError(N.GEO_ERR_INVALID_ARG, "Mesh must have stress_history")
    out = np.empty((mesh.num_elements(), 6))
    sn = np.ascontiguousarray(mesh.stress_history.stress, np.float64)
    ctx.check(N.lib().geo_update_stresses_maxwell(ctx.h, mesh.handle(ctx), material.youngs_modulus,
                                                  material.poisson_ratio, material.viscosity, _ptr(_f64(u_n)),
                                                  _ptr(_f64(u_next)), float(dt), _ptr(sn), _ptr(out)))
    return out


@dataclass
class TimeStepStats:
    """time_integration.rs:11-20."""
    time: float
    dt: float
    iterations: int
    residual: float


class BackwardEuler:
    """time_integration.rs:38-160: backward Euler for Maxwell viscoelasticity.

    ``step`` follows the reference (assemble K_eff and f_history, add f_ext, apply
    the Dirichlet BCs, solve). ``step_operator`` takes the same step with a
    resident matrix-free ElasticityOperator (the elastic K does not change between
    steps), so nothing is re-assembled."""

    def __init__(self, n_dofs: int, dt: float):
        if not dt > 0:
            raise GeoError(N.GEO_ERR_INVALID_ARG, f"Time step must be positive, got {dt}")
        if not n_dofs > 0:
            raise GeoError(N.GEO_ERR_INVALID_ARG, f"Number of DOFs must be positive, got {n_dofs}")
        self.time, self.dt = 0.0, float(dt)
        self.displacement = np.zeros(int(n_dofs))

    @staticmethod
    def new(n_dofs, dt):
        return BackwardEuler(n_dofs, dt)

    def step(self, mesh: Mesh, dof_mgr: DofManager, material: MaxwellViscoelasticity, f_ext, solver):
        K, f_hist = Assembler.assemble_maxwell_viscoelastic_parallel(mesh, dof_mgr, material, self.dt)
        Kb, fb = Assembler.apply_dirichlet_bcs(K, np.asarray(f_ext, np.float64) + f_hist, dof_mgr)
        u, st = solver.solve(Kb, fb)
        return self._advance(u, st)

    def step_operator(self, op: "ElasticityOperator", mesh: Mesh, f_ext, solver):
        f_hist = Assembler.maxwell_history_force(mesh, mesh.stress_history, op.ctx)
        u, st = op.forward(np.asarray(f_ext, np.float64) + f_hist, solver)
        return self._advance(u, st)

    def _advance(self, u, st):
        self.displacement = u
        self.time += self.dt
        return u, TimeStepStats(self.time, self.dt, st.iterations, st.residual_norm)

    def current_time(self):
        return self.time

    def current_displacement(self):
        return self.displacement

    def reset(self):
        self.time = 0.0
        self.displacement = np.zeros_like(self.displacement)

    def set_timestep(self, dt):
        if not dt > 0:
            raise GeoError(N.GEO_ERR_INVALID_ARG, f"Time step must be positive, got {dt}")
        self.dt = float(dt)


# --------------------------------------------------------------------------- solvers
@dataclass
class SolverStats:
    """solver.rs:5-20 plus extensions."""
    iterations: int = 0
    residual_norm: float = 0.0
    relative_residual: float = 0.0
    converged: bool = False
    solve_time: float = 0.0
    status: int = 0
    fp64_residual_updates: int = 0
    b_norm: float = 0.0
    kernel_launches: int = 0

    @classmethod
    def from_c(cls, s: N.SolverStatsC):
        return cls(int(s.iterations), float(s.residual_norm), float(s.relative_residual), bool(s.converged),
                   float(s.solve_time), int(s.status), int(s.fp64_residual_updates), float(s.b_norm),
                   int(s.kernel_launches))


class _CsrKrylov:
    """Shared builder API of BiCGSTAB and GMRES (iterative.rs:150-175, :303-331)."""

    def __init__(self, name):
        self.max_iterations = 1000
        self.tolerance = 1e-8
        self.abs_tolerance = 1e-12
        self.use_preconditioner = True
        self.verbose = False
        self.timeout_seconds = 10.0
        self.name = name

    def with_max_iterations(self, n):
        self.max_iterations = int(n)
        return self

    def with_tolerance(self, t):
        self.tolerance = float(t)
        return self

    def with_abs_tolerance(self, t):
        self.abs_tolerance = float(t)
        return self

    def with_verbose(self, flag):
        self.verbose = bool(flag)  # progress printing is not mirrored
        return self

    def with_preconditioner(self, flag):
        self.use_preconditioner = bool(flag)
        return self

    def opts(self) -> N.CgOpts:
        o = N.default_opts()
        o.max_iterations = self.max_iterations
        o.tolerance = self.tolerance
        o.abs_tolerance = self.abs_tolerance
        o.use_preconditioner = int(self.use_preconditioner)
        o.timeout_seconds = self.timeout_seconds
        return o

    def _solve(self, fn, A, b, *extra):
        b = _f64(b)
        x = np.empty(A.rows()) if isinstance(b, np.ndarray) else b.new_empty(A.rows())
        st = N.SolverStatsC()
        o = self.opts()
        A.ctx.check(fn(A.ctx.h, A.h, _ptr(b), C.byref(o), *extra, _ptr(x), C.byref(st)),
                    allow=(N.GEO_NOT_CONVERGED, N.GEO_ERR_BREAKDOWN))
        return x, SolverStats.from_c(st)


class BiCGSTAB(_CsrKrylov):
    """iterative.rs:150-301: right-preconditioned BiCGSTAB on the GPU (FP64, CSR)."""

    def __init__(self):
        super().__init__("BiCGSTAB")

    new = classmethod(lambda cls: cls())

    def solve(self, A: "CsrMatrix", b):
        """Solver::solve (iterative.rs:281-288). Returns (x, SolverStats)."""
        return self._solve(N.lib().geo_bicgstab_solve, A, b)


class GMRES(_CsrKrylov):
    """iterative.rs:303-479: restarted, right-preconditioned GMRES on the GPU (FP64, CSR)."""

    def __init__(self):
        super().__init__("GMRES")
        self.restart = 10

    new = classmethod(lambda cls: cls())

    def with_restart(self, m):
        self.restart = int(m)
        return self

    def solve(self, A: "CsrMatrix", b):
        """Solver::solve (iterative.rs:459-466). Returns (x, SolverStats)."""
        return self._solve(N.lib().geo_gmres_solve, A, b, self.restart)


class DirectSolver:
    """direct.rs:9-95: dense LU with partial pivoting on the GPU (FP64); no iterations."""

    def __init__(self):
        self.name = "Direct (Sparse LU)"

    new = classmethod(lambda cls: cls())

    def solve(self, A: "CsrMatrix", b):
        """Solver::solve (direct.rs:28-73). Returns (x, SolverStats); a singular
        matrix raises GeoError(GEO_ERR_SINGULAR_MATRIX), where the reference panics."""
        b = _f64(b)
        x = np.empty(A.rows()) if isinstance(b, np.ndarray) else b.new_empty(A.rows())
        st = N.SolverStatsC()
        A.ctx.check(N.lib().geo_direct_solve(A.ctx.h, A.h, _ptr(b), _ptr(x), C.byref(st)))
        return x, SolverStats.from_c(st)

    def solve_with_operator(self, A, b, precond=None):
        """direct.rs:75-86: the direct solver needs an assembled matrix."""
        raise N.GeoError(N.GEO_ERR_UNSUPPORTED,
                         "DirectSolver does not support matrix-free operator. Use iterative solvers instead.")

    # direct.rs:92-95: the tolerances are fixed at 0 and the setters do nothing
    def tolerance(self):
        return 0.0

    def abs_tolerance(self):
        return 0.0

    def set_tolerance(self, t):
        pass

    def set_abs_tolerance(self, t):
        pass


class ConjugateGradient:
    """iterative.rs:7-147: Jacobi-preconditioned CG with the builder API."""

    def __init__(self):
        self.max_iterations = 1000
        self.tolerance = 1e-8
        self.abs_tolerance = 1e-12
        self.use_preconditioner = True
        self.precision = N.PRECISION_FP64
        self.reliable_delta = 0.1
        self.timeout_seconds = 10.0
        self.name = "ConjugateGradient"

    @staticmethod
    def new():
        return ConjugateGradient()

    def with_max_iterations(self, n):
        self.max_iterations = int(n)
        return self

    def with_tolerance(self, t):
        self.tolerance = float(t)
        return self

    def with_abs_tolerance(self, t):
        self.abs_tolerance = float(t)
        return self

    def with_preconditioner(self, flag):
        self.use_preconditioner = bool(flag)
        return self

    def with_precision(self, precision):
        """'fp64' (default, the reference semantics) or 'mixed' (matrix-free only)."""
        self.precision = {"fp64": N.PRECISION_FP64, "mixed": N.PRECISION_MIXED}.get(precision, precision)
        return self

    def opts(self) -> N.CgOpts:
        o = N.default_opts()
        o.max_iterations = self.max_iterations
        o.tolerance = self.tolerance
        o.abs_tolerance = self.abs_tolerance
        o.use_preconditioner = int(self.use_preconditioner)
        o.precision = int(self.precision)
        o.reliable_delta = self.reliable_delta
        o.timeout_seconds = self.timeout_seconds
        return o

    def solve(self, A: CsrMatrix, b):
        """Solver::solve (iterative.rs:123-131). Returns (x, SolverStats)."""
        b = _f64(b)
        x = np.empty(A.rows()) if isinstance(b, np.ndarray) else b.new_empty(A.rows())
        st = N.SolverStatsC()
        o = self.opts()
        A.ctx.check(N.lib().geo_cg_solve(A.ctx.h, A.h, _ptr(b), C.byref(o), _ptr(x), C.byref(st)),
                    allow=(N.GEO_NOT_CONVERGED, N.GEO_ERR_BREAKDOWN))
        return x, SolverStats.from_c(st)

    def solve_with_operator(self, op: "_MatFreeOperator", b):
        """Solver::solve_with_operator (solver.rs:112-120) for a matrix-free operator."""
        return op.solve(b, self)


# --------------------------------------------------------------------------- matrix-free
class _MatFreeOperator:
    _create = None

    def _init(self, mesh, dof_mgr, ctx, h):
        self.mesh, self.dof_mgr, self.ctx, self.h = mesh, dof_mgr, ctx, h
        nd, ne, cd = C.c_int64(), C.c_int64(), C.c_double()
        N.check(N.lib().geo_op_info(h, C.byref(nd), C.byref(ne), C.byref(cd)))
        self.n_dofs, self.n_elem, self.char_diag = nd.value, ne.value, cd.value

    def rows(self):
        return self.n_dofs

    cols = rows

    def _out(self, like, n):
        return np.empty(n) if isinstance(like, np.ndarray) else like.new_empty(n)

    def set_coefficients(self, coef):
        p, k, keep = _coef_ptr(coef, self.n_elem)
        self.ctx.check(N.lib().geo_op_set_coefficients(self.h, p, k))
        cd = C.c_double()
        N.check(N.lib().geo_op_info(self.h, None, None, C.byref(cd)))
        self.char_diag = cd.value

    def apply(self, x, precision="fp64"):
        x = _f64(x)
        y = self._out(x, self.n_dofs)
        prec = N.PRECISION_MIXED if precision == "mixed" else N.PRECISION_FP64
        self.ctx.check(N.lib().geo_op_apply(self.h, _ptr(x), _ptr(y), prec))
        return y

    def lift_rhs(self, f):
        f = _f64(f)
        out = self._out(f, self.n_dofs)
        self.ctx.check(N.lib().geo_op_lift_rhs(self.h, _ptr(f), _ptr(out)))
        return out

    def diagonal(self):
        d = np.empty(self.n_dofs)
        self.ctx.check(N.lib().geo_op_diagonal(self.h, _ptr(d)))
        return d

    def solve(self, b, solver: ConjugateGradient | None = None):
        solver = solver or ConjugateGradient()
        b = _f64(b)
        x = self._out(b, self.n_dofs)
        st = N.SolverStatsC()
        o = solver.opts()
        self.ctx.check(N.lib().geo_cg_solve_matfree(self.h, _ptr(b), C.byref(o), _ptr(x), C.byref(st)),
                       allow=(N.GEO_NOT_CONVERGED, N.GEO_ERR_BREAKDOWN))
        return x, SolverStats.from_c(st)

    def forward(self, f, solver: ConjugateGradient | None = None):
        solver = solver or ConjugateGradient()
        f = _f64(f)
        u = self._out(f, self.n_dofs)
        st = N.SolverStatsC()
        o = solver.opts()
        self.ctx.check(N.lib().geo_forward(self.h, _ptr(f), C.byref(o), _ptr(u), C.byref(st)),
                       allow=(N.GEO_NOT_CONVERGED,))
        return u, SolverStats.from_c(st)

    def vjp(self, dJ_du, u=None, f=None, solver: ConjugateGradient | None = None):
        """dJ/d(ln coef_e) given dJ/du; u=None recomputes the forward solution from f."""
        solver = solver or ConjugateGradient()
        g = _f64(dJ_du)
        out = self._out(g, self.n_elem)
        st = N.SolverStatsC()
        o = solver.opts()
        uu = None if u is None else _f64(u)
        ff = None if f is None else _f64(f)
        self.ctx.check(N.lib().geo_vjp(self.h, _ptr(ff), _ptr(uu), _ptr(g), C.byref(o), _ptr(out), C.byref(st)),
                       allow=(N.GEO_NOT_CONVERGED,))
        return out, SolverStats.from_c(st)

    def element_gradient(self, u, lam):
        u, lam = _f64(u), _f64(lam)
        out = self._out(u, self.n_elem)
        self.ctx.check(N.lib().geo_op_element_gradient(self.h, _ptr(u), _ptr(lam), _ptr(out)))
        return out

    def __del__(self):
        try:
            N.lib().geo_op_destroy(self.h)
        except Exception:
            pass


class ThermalOperator(_MatFreeOperator):
    """Matrix-free K_bc of apply_dirichlet_bcs(assemble_thermal_stiffness_parallel(..))."""

    def __init__(self, mesh: Mesh, dof_mgr: DofManager, conductivity, ctx=None):
        ctx = _ctx(ctx)
        p, k, keep = _coef_ptr(conductivity, mesh.num_elements())
        h = C.c_void_p()
        ctx.check(N.lib().geo_thermal_operator_create(ctx.h, mesh.handle(ctx), dof_mgr.handle(ctx), p, k,
                                                      C.byref(h)))
        self._init(mesh, dof_mgr, ctx, h)


class ElasticityOperator(_MatFreeOperator):
    """Matrix-free K_bc of the 3-DOF elasticity system (assembly.rs:389-437 + :168-230)."""

    def __init__(self, mesh: Mesh, dof_mgr: DofManager, material: IsotropicElasticity, youngs_e=None, ctx=None):
        ctx = _ctx(ctx)
        ee = None if youngs_e is None else _f64(youngs_e)
        h = C.c_void_p()
        ctx.check(N.lib().geo_elasticity_operator_create(ctx.h, mesh.handle(ctx), dof_mgr.handle(ctx), _ptr(ee),
                                                         float(material.youngs_modulus),
                                                         float(material.poisson_ratio), C.byref(h)))
        self._init(mesh, dof_mgr, ctx, h)
