"""Coefficient updates on an existing operator (ThermalOperator.set_coefficients).

The patch kernels scale each patch's fixed-point sums by a bound built from the
element coefficients, and read it, with the patch's sizes, from a per-patch
record. An update must rebuild both: with a bound left 1000 times too small the
INT32 sums would overflow. The solves after a 1000-fold increase and a 1000-fold
decrease of k must match the oracle's CG on the same systems (assemble_thermal_
stiffness, apply_dirichlet_bcs, cg_solve: the reference's assembly.rs and
iterative.rs), in FP64 and in mixed precision."""
import numpy as np
import pytest

from conftest import thermal_problem


@pytest.mark.gpu
def test_set_coefficients_rebuilds_patch_bounds(orc, geo):
    xyz, conn, mask, vals = thermal_problem(10, orc)
    rng = np.random.default_rng(77)
    k0 = np.exp(np.log(3.0) + 0.5 * rng.normal(size=conn.shape[0]))
    mesh = geo.Mesh(xyz, conn)
    dm = geo.DofManager(xyz.shape[0], 1)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, vals[idx])
    fg = geo.Assembler.assemble_thermal_load(mesh, dm, 1e-6)
    f = orc.assemble_thermal_load(xyz, conn, 1e-6)
    op = geo.ThermalOperator(mesh, dm, k0)
    for scale in (1.0, 1e3, 1e-3):
        k = k0 * scale
        if scale != 1.0:
            op.set_coefficients(k)
        K = orc.assemble_thermal_stiffness(xyz, conn, k_e=k)
        Kbc, fbc = orc.apply_dirichlet_bcs(K, f, mask, vals)
        ref, _ = orc.cg_solve(Kbc, fbc, max_iterations=20000, tolerance=1e-12)
        for prec in ("fp64", "mixed"):
            solver = geo.ConjugateGradient().with_tolerance(1e-10).with_max_iterations(20000).with_precision(prec)
            u, st = op.forward(fg, solver)
            assert st.converged, (scale, prec)
            assert np.all(np.isfinite(u)), (scale, prec)
            assert np.linalg.norm(u - ref) <= 1e-8 * np.linalg.norm(ref), (scale, prec)
