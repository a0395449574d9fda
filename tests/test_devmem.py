"""The library's caching device allocator (no reference counterpart): objects
created and destroyed call after call reuse the device memory of earlier ones,
results do not depend on it, and geo_release_cached_memory returns the kept
memory to the driver."""
import numpy as np
import pytest

from conftest import thermal_problem


def test_release_symbol_is_exported():
    from geo_simulator_b200 import _native as N
    assert hasattr(N.lib(), "geo_release_cached_memory")


@pytest.mark.gpu
def test_reuse_across_create_destroy_and_release(orc, geo):
    import torch
    from geo_simulator_b200 import _native as N
    xyz, conn, mask, vals = thermal_problem(20, orc)
    mesh = geo.Mesh(xyz, conn)
    rng = np.random.default_rng(3)
    k_e = np.exp(np.log(3.0) + 0.5 * rng.normal(size=conn.shape[0]))
    solver = geo.ConjugateGradient().with_tolerance(1e-10).with_max_iterations(20000)
    us = []
    for _ in range(3):  # objects of the same sizes: the later ones run on cached blocks
        dm = geo.DofManager(xyz.shape[0], 1)
        idx = np.nonzero(mask)[0]
        dm.set_dirichlet(idx, vals[idx])
        op = geo.ThermalOperator(mesh, dm, k_e)
        f = geo.Assembler.assemble_thermal_load(mesh, dm, 1e-6)
        u, st = op.forward(f, solver)
        assert st.converged
        us.append(u)
        del op
    for u in us[1:]:
        assert np.linalg.norm(u - us[0]) <= 1e-9 * np.linalg.norm(us[0])
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    assert N.lib().geo_release_cached_memory() == 0
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after >= free_before
