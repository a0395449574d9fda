"""geo_cg_solve_noalloc (no reference counterpart): the allocation-free CSR PCG
against geo_cg_solve on the same system, on two calls in a row (the second call
checks that the barrier word and result slot start from zero again), plus its
size and pointer checks. The file name sorts last so that it runs after every
other GPU test in a full session; it also passes alone."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _thermal_system(orc, geo, n=6):
    mesh = geo.ImprovedMeshGenerator.generate_cube(n, n, n, 1000.0, 1000.0, 600.0)
    mask, vals = orc.thermal_bc(mesh.nodes, 600.0)
    d = geo.DofManager(mesh.num_nodes(), 1)
    d.set_dirichlet(np.nonzero(mask)[0], vals[mask == 1])
    K = geo.Assembler.assemble_thermal_stiffness_parallel(mesh, d, 3.0)
    f = geo.Assembler.assemble_thermal_load(mesh, d, 1e-6)
    return geo.Assembler.apply_dirichlet_bcs(K, f, d)


def _noalloc(geo, A, b_ptr, x_ptr, solver):
    from geo_simulator_b200 import _native as N
    st = N.SolverStatsC()
    o = solver.opts()
    code = N.lib().geo_cg_solve_noalloc(A.ctx.h, A.h, b_ptr, C.byref(o), x_ptr, C.byref(st))
    return code, st


def _mallocs():
    from geo_simulator_b200 import _native as N
    live, cached, n = C.c_int64(), C.c_int64(), C.c_int64()
    assert N.lib().geo_device_memory_stats(C.byref(live), C.byref(cached), C.byref(n)) == N.GEO_OK
    return live.value, cached.value, n.value


def test_noalloc_matches_cg_solve_on_two_calls(orc, geo):
    import torch
    from geo_simulator_b200 import _native as N
    Kb, fb = _thermal_system(orc, geo)
    solver = geo.ConjugateGradient().with_tolerance(1e-10)
    x_ref, st_ref = solver.solve(Kb, fb)
    assert st_ref.converged
    b = torch.from_numpy(fb).cuda()
    xs = [torch.full_like(b, float("nan")) for _ in range(2)]
    for call in range(2):
        x = xs[call]
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        stats0 = _mallocs()
        code, st = _noalloc(geo, Kb, b.data_ptr(), x.data_ptr(), solver)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        stats1 = _mallocs()
        assert code == N.GEO_OK, N.lib().geo_last_error(Kb.ctx.h)
        # same kernel, same grid, fixed-order reductions: bit-identical
        assert np.array_equal(x.cpu().numpy(), x_ref), call
        assert st.iterations == st_ref.iterations and st.converged == 1
        assert st.residual_norm == st_ref.residual_norm
        if call == 1:
            # the call after the first takes no device memory: the driver's free
            # memory and the library allocator's counters are unchanged across it
            assert free1 == free0, (free0, free1)
            assert stats1 == stats0, (stats0, stats1)


def test_noalloc_not_converged_matches(orc, geo):
    import torch
    from geo_simulator_b200 import _native as N
    Kb, fb = _thermal_system(orc, geo, 4)
    solver = geo.ConjugateGradient().with_max_iterations(3)
    x_ref, _ = solver.solve(Kb, fb)
    b = torch.from_numpy(fb).cuda()
    x = torch.empty_like(b)
    code, st = _noalloc(geo, Kb, b.data_ptr(), x.data_ptr(), solver)
    assert code == N.GEO_NOT_CONVERGED and st.iterations == 3
    assert np.array_equal(x.cpu().numpy(), x_ref)


def test_noalloc_rejects_oversize_and_host_pointers(orc, geo):
    import torch
    from geo_simulator_b200 import _native as N
    big = 262144 + 1
    idx = np.arange(big)
    A = geo.CsrMatrix.from_triplets(big, big, idx, idx, np.ones(big))
    b = torch.ones(big, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    code, _ = _noalloc(geo, A, b.data_ptr(), x.data_ptr(), geo.ConjugateGradient())
    assert code == N.GEO_ERR_INVALID_ARG
    assert "GEO_NOALLOC_MAX_ROWS" in N.lib().geo_last_error(A.ctx.h).decode()
    Kb, fb = _thermal_system(orc, geo, 2)
    xh = np.empty_like(fb)
    code, _ = _noalloc(geo, Kb, fb.ctypes.data, xh.ctypes.data, geo.ConjugateGradient())
    assert code == N.GEO_ERR_INVALID_ARG
    assert "device memory" in N.lib().geo_last_error(Kb.ctx.h).decode()
