"""ImprovedMeshGenerator::generate_cube (mesh_generator_improved.rs:19-169) on the
device: ``geo_mesh_generate_cube`` builds the SoA device mesh directly.

CPU: the host generator against the oracle's restatement (the reference's
HashMap first-touch numbering) and the entry points' exports.
GPU: the device mesh, copied out, equals the host generator and the oracle bit
for bit (coordinates compared as IEEE bit patterns) on lopsided, degenerate and
mirrored boxes; a device mesh assembles the same CSR as the uploaded host mesh;
argument errors."""
import ctypes as C

import numpy as np
import pytest

SHAPES = [
    (1, 1, 1, 1.0, 1.0, 1.0),
    (2, 3, 4, 1000.0, 800.0, 600.0),
    (5, 1, 2, 0.7, 1.3, 2.9),
    (3, 4, 2, 1e-3, 7.0, 1e5),
    (5, 2, 3, -1.0, 2.0, 0.5),  # mirrored: every orientation swap flips
    (2, 2, 2, 0.0, 1.0, 1.0),  # flat: zero determinants, no swaps
    (7, 6, 5, 1000.0, 1000.0, 600.0),
]


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


# ------------------------------------------------------------------------ CPU
def test_host_generator_matches_oracle(orc, geo):
    for s in SHAPES:
        xyz, conn = orc.generate_cube(*s)
        m = geo.ImprovedMeshGenerator.generate_cube(*s)
        assert np.array_equal(m.elements, conn)
        assert np.array_equal(_bits(m.nodes), _bits(xyz))


def test_device_generator_exports(geo):
    from geo_simulator_b200 import _native as N
    lib = N.lib()
    for name in ("geo_mesh_generate_cube", "geo_mesh_size", "geo_mesh_download"):
        assert hasattr(lib, name)
    # size query on a NULL mesh is an argument error, not a crash
    n = C.c_int64()
    assert lib.geo_mesh_size(None, C.byref(n), None) == N.GEO_ERR_INVALID_ARG


# ------------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
def test_device_mesh_bit_exact(orc, geo, shape):
    xyz, conn = orc.generate_cube(*shape)
    dm = geo.ImprovedMeshGenerator.generate_cube_device(*shape)
    assert dm.num_nodes() == xyz.shape[0] and dm.num_elements() == conn.shape[0]
    assert np.array_equal(dm.elements, conn)
    assert np.array_equal(_bits(dm.nodes), _bits(xyz))


@pytest.mark.gpu
def test_device_mesh_bit_exact_large(geo):
    s = (48, 40, 32, 1000.0, 1000.0, 600.0)
    hm = geo.ImprovedMeshGenerator.generate_cube(*s)
    dm = geo.ImprovedMeshGenerator.generate_cube_device(*s)
    assert np.array_equal(dm.elements, hm.elements)
    assert np.array_equal(_bits(dm.nodes), _bits(hm.nodes))


@pytest.mark.gpu
def test_device_mesh_download_to_device_buffers(geo):
    import torch
    s = (6, 5, 4, 3.0, 2.0, 1.0)
    hm = geo.ImprovedMeshGenerator.generate_cube(*s)
    dm = geo.ImprovedMeshGenerator.generate_cube_device(*s)
    from geo_simulator_b200 import _native as N
    xyz = torch.empty((dm.num_nodes(), 3), dtype=torch.float64, device="cuda")
    conn = torch.empty((dm.num_elements(), 10), dtype=torch.int32, device="cuda")
    h = dm.handle()
    torch.cuda.synchronize()
    N.check(N.lib().geo_mesh_download(h, C.c_void_p(xyz.data_ptr()), C.c_void_p(conn.data_ptr())))
    assert np.array_equal(conn.cpu().numpy(), hm.elements)
    assert np.array_equal(_bits(xyz.cpu().numpy()), _bits(hm.nodes))


@pytest.mark.gpu
def test_device_mesh_assembles_like_host_mesh(geo):
    s = (6, 6, 4, 1000.0, 1000.0, 600.0)
    hm = geo.ImprovedMeshGenerator.generate_cube(*s)
    dm = geo.ImprovedMeshGenerator.generate_cube_device(*s)
    dofs = geo.DofManager(hm.num_nodes(), 1)
    Kh = geo.Assembler.assemble_thermal_stiffness_parallel(hm, dofs, 2.5).to_host()
    Kd = geo.Assembler.assemble_thermal_stiffness_parallel(dm, dofs, 2.5).to_host()
    for a, b in zip(Kh, Kd):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    # the device mesh was used without copying its arrays to the host
    assert dm._nodes is None and dm._elements is None


@pytest.mark.gpu
def test_device_generator_rejects_bad_sizes(geo):
    for bad in ((0, 1, 1), (1, -2, 1), (1, 1, 0)):
        with pytest.raises(geo.GeoError):
            geo.ImprovedMeshGenerator.generate_cube_device(*bad, 1.0, 1.0, 1.0)
    with pytest.raises(geo.GeoError):  # node ids would overflow int32
        geo.ImprovedMeshGenerator.generate_cube_device(1 << 11, 1 << 11, 1 << 10, 1.0, 1.0, 1.0)
