"""The three ways the PCG's patch kernel hands shared-node contributions
to the node update: red.global.add (mode 0), halo slots carried in shared memory
(1) and halo slots read from global memory (2). The operator set-up picks one
by occupancy (2 only on large meshes); GEO_PATCH_HALO forces each here, and the
solutions must agree with the oracle's CG and with each other, in FP64 and mixed
precision. The node counts are not multiples of the node update's vector width,
so its scalar tail runs too. GEO_PATCH_NBUF=1 forces the single-buffer patch
kernel (taken when two element-data buffers exceed shared memory); with halo
slots its sums are the same fixed-point sums in the same order, so its solutions
must equal the double-buffer kernel's bit for bit."""
import os

import numpy as np
import pytest

from conftest import thermal_problem


def same_sums(u, it, other, mode):
    """Single- against double-buffer kernel: bit for bit in the halo-slot modes;
    mode 0's red.global.add sums shared nodes in arrival order."""
    u2, it2 = other
    if mode == "0":
        assert np.linalg.norm(u - u2) <= 1e-9 * np.linalg.norm(u2)
    else:
        assert np.array_equal(u, u2), mode
        assert it == it2, mode


@pytest.mark.gpu
@pytest.mark.parametrize("n", [7, 12])
def test_halo_modes_agree(orc, geo, n, monkeypatch):
    xyz, conn, mask, vals = thermal_problem(n, orc)
    rng = np.random.default_rng(n)
    k_e = np.exp(np.log(3.0) + 0.5 * rng.normal(size=conn.shape[0]))
    K = orc.assemble_thermal_stiffness(xyz, conn, k_e=k_e)
    f = orc.assemble_thermal_load(xyz, conn, 1e-6)
    Kbc, fbc = orc.apply_dirichlet_bcs(K, f, mask, vals)
    ref, _ = orc.cg_solve(Kbc, fbc, max_iterations=20000, tolerance=1e-12)
    mesh = geo.Mesh(xyz, conn)
    dm = geo.DofManager(xyz.shape[0], 1)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, vals[idx])
    fg = geo.Assembler.assemble_thermal_load(mesh, dm, 1e-6)
    sols = {}
    for nbuf in ("2", "1"):
        monkeypatch.setenv("GEO_PATCH_NBUF", nbuf)
        for mode in ("0", "1", "2"):
            monkeypatch.setenv("GEO_PATCH_HALO", mode)
            op = geo.ThermalOperator(mesh, dm, k_e)
            for prec in ("fp64", "mixed"):
                solver = geo.ConjugateGradient().with_tolerance(1e-10).with_max_iterations(20000).with_precision(prec)
                u, st = op.forward(fg, solver)
                assert st.converged, (mode, prec)
                assert np.linalg.norm(u - ref) <= 1e-8 * np.linalg.norm(ref), (mode, prec)
                if nbuf == "2":
                    sols[mode, prec] = (u, st.iterations)
                else:
                    same_sums(u, st.iterations, sols[mode, prec], mode)
            del op
    for prec in ("fp64", "mixed"):
        u0, it0 = sols["0", prec]
        for mode in ("1", "2"):
            u, it = sols[mode, prec]
            assert np.linalg.norm(u - u0) <= 1e-9 * np.linalg.norm(u0)
            assert abs(it - it0) <= 3


@pytest.mark.gpu
def test_halo_modes_agree_elasticity(orc, geo, monkeypatch):
    """The same for 3-DOF elasticity (gravity on a half-space): every mode against
    the oracle's CG on K_bc, run to rel-res 1e-13."""
    from test_gpu_elasticity import halfspace, setup
    xyz, conn, mask, vals, E_e = halfspace(orc, 8, 7, 5)
    mesh, d = setup(geo, xyz, conn, mask, vals)
    mat = geo.IsotropicElasticity(1e11, 0.25)
    Ko = orc.assemble_elasticity_stiffness(xyz, conn, E_e=E_e, nu=0.25)
    fo = orc.assemble_gravity_load(xyz, conn, 3300.0, [0, 0, -9.81])
    Kbo, fbo = orc.apply_dirichlet_bcs(Ko, fo, mask, vals)
    ul, _ = orc.cg_solve(Kbo, fbo, max_iterations=50000, tolerance=1e-13)
    sols = {}
    for nbuf in ("2", "1"):
        monkeypatch.setenv("GEO_PATCH_NBUF", nbuf)
        for mode in ("0", "1", "2"):
            monkeypatch.setenv("GEO_PATCH_HALO", mode)
            op = geo.ElasticityOperator(mesh, d, mat, E_e)
            for prec in ("fp64", "mixed"):
                solver = geo.ConjugateGradient().with_max_iterations(20000).with_tolerance(1e-10).with_precision(prec)
                u, st = op.solve(fbo, solver)
                assert st.converged, (mode, prec)
                assert np.linalg.norm(u - ul) <= 1e-8 * np.linalg.norm(ul), (mode, prec)
                if nbuf == "2":
                    sols[mode, prec] = (u, st.iterations)
                else:
                    same_sums(u, st.iterations, sols[mode, prec], mode)
            del op
    for prec in ("fp64", "mixed"):
        u0, it0 = sols["0", prec]
        for mode in ("1", "2"):
            u, it = sols[mode, prec]
            assert np.linalg.norm(u - u0) <= 1e-9 * np.linalg.norm(u0)
            assert abs(it - it0) <= 5
