"""Failure detection without faulting the GPU: bounded device waits that run out
and report GEO_ERR_TIMEOUT, reference panics turned into status codes, and the
reference's solver edge cases (iterative.rs:60-68, :85, non-convergence)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_barrier_timeout_is_reported_and_context_survives(geo):
    from geo_simulator_b200 import _native as N
    ctx = geo.Context.default()
    code = N.lib().geo_debug_barrier_timeout(ctx.h, 0.2)
    assert code == N.GEO_ERR_TIMEOUT
    assert "timed out" in N.lib().geo_last_error(ctx.h).decode()
    # the context is still usable
    A = geo.CsrMatrix.from_triplets(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [2.0, 1.0, 1.0, 2.0])
    x, st = geo.ConjugateGradient().solve(A, np.array([3.0, 3.0]))
    assert st.converged and np.abs(x - 1.0).max() < 1e-6


def test_cg_2x2_and_diagonal_jacobi(geo):
    """iterative.rs:490-504 and preconditioner.rs:212-230."""
    A = geo.CsrMatrix.from_triplets(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [2.0, 1.0, 1.0, 2.0])
    x, st = geo.ConjugateGradient().solve(A, np.array([3.0, 3.0]))
    assert st.converged and np.abs(x - 1.0).max() < 1e-6
    D = geo.CsrMatrix.from_triplets(3, 3, [0, 1, 2], [0, 1, 2], [2.0, 4.0, 8.0])
    x, st = geo.ConjugateGradient().solve(D, np.array([2.0, 4.0, 8.0]))
    assert st.converged and st.iterations == 0 and np.abs(x - 1.0).max() < 1e-14
    assert np.allclose(D.apply(np.ones(3)), [2.0, 4.0, 8.0])


def test_zero_rhs_returns_zero(geo):
    """iterative.rs:60-68: ||b|| < 1e-25 -> zeros, converged, 0 iterations."""
    A = geo.CsrMatrix.from_triplets(2, 2, [0, 1], [0, 1], [1.0, 1.0])
    x, st = geo.ConjugateGradient().solve(A, np.zeros(2))
    assert st.converged and st.iterations == 0 and np.all(x == 0)


def test_breakdown_is_reported(geo):
    """iterative.rs:85: |p^T A p| < 1e-30 stops the loop, converged = false."""
    from geo_simulator_b200 import _native as N
    A = geo.CsrMatrix.from_triplets(2, 2, [0, 1], [0, 1], [0.0, 0.0])
    x, st = geo.ConjugateGradient().solve(A, np.array([1.0, 1.0]))
    assert not st.converged and st.status == N.GEO_ERR_BREAKDOWN


def test_not_converged_keeps_the_iterate(orc, geo):
    from geo_simulator_b200 import _native as N
    mesh = geo.ImprovedMeshGenerator.generate_cube(4, 4, 4, 1000.0, 1000.0, 600.0)
    mask, vals = orc.thermal_bc(mesh.nodes, 600.0)
    d = geo.DofManager(mesh.num_nodes(), 1)
    d.set_dirichlet(np.nonzero(mask)[0], vals[mask == 1])
    K = geo.Assembler.assemble_thermal_stiffness_parallel(mesh, d, 3.0)
    f = geo.Assembler.assemble_thermal_load(mesh, d, 1e-6)
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, f, d)
    x, st = geo.ConjugateGradient().with_max_iterations(3).solve(Kb, fb)
    assert not st.converged and st.iterations == 3 and st.status == N.GEO_NOT_CONVERGED
    assert np.isfinite(x).all() and np.abs(x).max() > 0
    op = geo.ThermalOperator(mesh, d, 3.0)
    for prec in ("fp64", "mixed"):
        xm, sm = op.solve(fb, geo.ConjugateGradient().with_max_iterations(3).with_precision(prec))
        assert not sm.converged and sm.status == N.GEO_NOT_CONVERGED and np.isfinite(xm).all()


def test_singular_jacobian_is_an_error(geo):
    """basis.rs:247 panics with 'Singular Jacobian'; here a status code."""
    nodes = np.zeros((10, 3))
    nodes[:, 0] = np.arange(10)  # all nodes on a line: det J = 0
    mesh = geo.Mesh(nodes, np.arange(10, dtype=np.int32).reshape(1, 10))
    with pytest.raises(geo.GeoError) as ei:
        geo.ElementMatrix.thermal_stiffness(mesh, 1.0)
    assert "Singular Jacobian" in str(ei.value)
    d = geo.DofManager(10, 1)
    with pytest.raises(geo.GeoError):
        geo.Assembler.assemble_thermal_stiffness_parallel(mesh, d, 1.0)
    with pytest.raises(geo.GeoError):
        geo.ThermalOperator(mesh, d, 1.0)


def test_invalid_arguments(geo):
    mesh = geo.ImprovedMeshGenerator.generate_cube(1, 1, 1, 1.0, 1.0, 1.0)
    with pytest.raises(geo.GeoError) as ei:
        geo.Assembler.assemble_elasticity_stiffness_parallel(mesh, geo.DofManager(mesh.num_nodes(), 1),
                                                            geo.IsotropicElasticity(1e9, 0.2))
    assert "3 DOF" in str(ei.value)
    with pytest.raises(geo.GeoError):
        geo.CsrMatrix.from_arrays(2, 2, np.array([0, 1, 2]), np.array([0, 5]), np.array([1.0, 1.0]))
    from geo_simulator_b200 import _native as N
    h = C.c_void_p()
    ctx = geo.Context.default()
    bad = np.arange(10, dtype=np.int32) + 100  # node ids beyond the node count
    assert N.lib().geo_mesh_create(ctx.h, 27, mesh.nodes.ctypes.data, 1, bad.ctypes.data, C.byref(h)) == \
        N.GEO_ERR_INVALID_ARG


def test_device_and_host_pointers_agree(geo, orc):
    import torch
    mesh = geo.ImprovedMeshGenerator.generate_cube(3, 3, 3, 1000.0, 1000.0, 600.0)
    mask, vals = orc.thermal_bc(mesh.nodes, 600.0)
    d = geo.DofManager(mesh.num_nodes(), 1)
    d.set_dirichlet(np.nonzero(mask)[0], vals[mask == 1])
    op = geo.ThermalOperator(mesh, d, 3.0)
    x = np.random.default_rng(0).standard_normal(mesh.num_nodes())
    yh = op.apply(x)
    yd = op.apply(torch.from_numpy(x).cuda())
    assert np.abs(yd.cpu().numpy() - yh).max() <= 1e-12 * np.abs(yh).max()
