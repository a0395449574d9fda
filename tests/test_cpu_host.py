"""CPU-side checks of the product: the C-ABI library loads and exports every
declared entry point, the host mesh generator matches the reference's numbering
bit for bit, the Python mirror's host logic, the seeded inputs, and the
multi-rank bench plumbing (gloo, world size 2). No GPU compute is called."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "geo_fem.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(geo_\w+)\s*\(", src, flags=re.M)))


def test_library_loads_and_exports_header_symbols():
    from geo_simulator_b200 import _native
    L = _native.lib()
    names = header_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_native.exported_symbols())
    assert L.geo_version().decode().startswith("geofem-b200")


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from geo_simulator_b200 import _native
    h = C.c_void_p()
    assert _native.lib().geo_ctx_create(0, C.byref(h)) == _native.GEO_ERR_NO_DEVICE


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 2, 2), (3, 4, 5), (6, 6, 6), (7, 2, 3), (5, 5, 1)])
def test_mesh_generator_bit_exact(orc, geo, dims):
    xyz, conn = orc.generate_cube(*dims, 1000.0, 1000.0, 600.0)
    m = geo.ImprovedMeshGenerator.generate_cube(*dims, 1000.0, 1000.0, 600.0)
    assert np.array_equal(m.nodes, xyz)
    assert np.array_equal(m.elements, conn)


def test_mesh_generator_sizes(geo):
    from geo_simulator_b200 import _native
    n, e = C.c_int64(), C.c_int64()
    assert _native.lib().geo_generate_cube_size(128, 128, 128, C.byref(n), C.byref(e)) == 0
    assert (n.value, e.value) == (16974593, 12582912)
    assert _native.lib().geo_generate_cube_size(64, 64, 64, C.byref(n), C.byref(e)) == 0
    assert (n.value, e.value) == (2146689, 1572864)
    assert _native.lib().geo_generate_cube_size(0, 1, 1, C.byref(n), C.byref(e)) == _native.GEO_ERR_INVALID_ARG


def test_dof_manager_semantics(geo):
    """dof.rs:37-155: dof = node * dpn + comp, Dirichlet set and counts."""
    d = geo.DofManager(5, 3)
    assert d.total_dofs() == 15 and d.global_dof(2, 1) == 7
    d.set_dirichlet_node(1, 2.5)
    d.set_dirichlet(d.global_dof(4, 2), -1.0)
    assert d.num_constrained_dofs() == 4 and d.num_free_dofs() == 11
    assert d.is_dirichlet(3) and d.is_dirichlet(14) and not d.is_dirichlet(0)
    assert d.get_dirichlet_value(4) == 2.5 and d.get_dirichlet_value(14) == -1.0
    with pytest.raises(geo.GeoError):
        d.global_dof(0, 3)


def test_material_validation(geo):
    with pytest.raises(geo.GeoError):
        geo.IsotropicElasticity(-1.0, 0.25)
    with pytest.raises(geo.GeoError):
        geo.IsotropicElasticity(1e9, 0.5)


def test_mesh_rejects_out_of_range_connectivity(geo):
    with pytest.raises(geo.GeoError):
        geo.Mesh(np.zeros((4, 3)), np.arange(10).reshape(1, 10))


def test_seeded_fields_are_deterministic():
    from geo_simulator_b200.fields import choice_distinct, lognormal_field, normal
    a = lognormal_field(1001, 1000, np.log(3.0), 0.5)
    b = lognormal_field(1001, 1000, np.log(3.0), 0.5)
    assert np.array_equal(a, b) and (a > 0).all()
    z = normal(7, 200000)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
    c = choice_distinct(2003, 5000, 1000)
    assert c.size == 1000 and np.unique(c).size == 1000 and c.max() < 5000


def test_bench_byte_and_flop_model():
    import bench
    from geo_simulator_b200 import kernel_timing as kt
    E, N = 12582912, 16974593
    # plain apply (int32 connectivity, k_e, coordinates): E(40 + 4) + N(12 + 4 + 4) + N/8
    assert bench.survey_apply_bytes(E, N, 4) == pytest.approx(E * 44 + N * 20 + N / 8)
    # PCG-mode patch launch, what it must move: 16-bit connectivity 20 B and G 6 x 4 B per
    # element, r / D^-1 / p_old in and p / q out per DOF, bitmask
    assert kt.patch_pcg_bytes(E, N, 4) == pytest.approx(E * 44 + N * 20 + N / 8)
    assert kt.patch_pcg_bytes(E, N, 8, 3) == pytest.approx(E * (20 + 80) + N * 3 * 40 + N / 8)
    assert kt.update_bytes(N, 4) == pytest.approx(28 * N + N / 8)
    # z-form of the mixed thermal solver: the patch kernel also moves x, the update only q, z, D^-1
    assert kt.patch_pcg_bytes(E, N, 4, zform=True) == pytest.approx(E * 44 + N * 24 + N / 8)
    assert kt.update_bytes(N, 4, zform=True) == pytest.approx(16 * N + N / 8)
    assert bench.solve_bytes(E, N, 10, 1) == pytest.approx(
        10 * (kt.patch_pcg_bytes(E, N, 4, zform=True) + kt.update_bytes(N, 4, zform=True)) + E * 68 + 16 * N + N / 8
        + 32 * N)
    # FLOPs per element from the kernels' formulation; CUDA-core peaks at 1965 MHz
    assert kt.patch_pcg_flops(E, N) == E * 216 + 3 * N
    assert kt.patch_pcg_flops(E, N, 3) == E * 1182 + 9 * N
    assert kt.cuda_core_peak_tflops(1965.0) == pytest.approx(74.45, rel=1e-3)
    assert kt.cuda_core_peak_tflops(1965.0, fp64=True) == pytest.approx(37.22, rel=1e-3)
    assert bench.cube_counts(128) == (12582912, 16974593)
    assert bench.cube_counts(48, 32) == (442368, 611585)


def test_reference_arm_loads_only_the_oracle():
    """The reference arm builds its inputs with the oracle's generate_cube: importing
    the package's numpy field helper must not load libgeofem.so."""
    import subprocess
    import sys
    code = ("import bench; xyz, conn, k, m, v = bench.oracle_inputs(2); "
            "maps = open('/proc/self/maps').read(); "
            "assert 'libgeofem' not in maps and 'liboracle' in maps; print(conn.shape[0])")
    out = subprocess.run([sys.executable, "-c", code], cwd=os.path.dirname(os.path.dirname(__file__)),
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "48"


def _gloo_worker(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    v = bench.max_over_ranks(1.0 + rank, dist, "cpu")
    bench.barrier(dist, "cpu")
    out[rank] = v
    dist.destroy_process_group()


def test_replica_timing_max_over_ranks_gloo():
    """bench.py reduces the timed region with MAX over ranks (replicas only)."""
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 2.0, 1: 2.0}
