"""Hand-written adjoint (no reference counterpart): element gradients against
the oracle's -lambda_e^T K_e u_e, and the full vector-Jacobian product against
central finite differences of FP64 forward solves and an FP64 CPU adjoint built
from the oracle's assembled CSR."""
import numpy as np
import pytest

from test_gpu_elasticity import halfspace, setup

pytestmark = pytest.mark.gpu


def thermal_setup(orc, geo, nx=6, ny=6, nz=4, sigma=0.3, seed=11):
    xyz, conn = orc.generate_cube(nx, ny, nz, 1000.0, 1000.0, 600.0)
    mask, vals = orc.thermal_bc(xyz, 600.0)
    lnk = np.log(3.0) + sigma * np.random.default_rng(seed).standard_normal(conn.shape[0])
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    d = geo.DofManager(xyz.shape[0], 1)
    idx = np.nonzero(mask)[0]
    d.set_dirichlet(idx, vals[idx])
    return xyz, conn, mask, vals, lnk, mesh, d


def test_element_gradient_matches_oracle(orc, geo):
    xyz, conn, mask, vals, lnk, mesh, d = thermal_setup(orc, geo, 3, 3, 2)
    op = geo.ThermalOperator(mesh, d, np.exp(lnk))
    rng = np.random.default_rng(3)
    u, lam = rng.standard_normal(xyz.shape[0]), rng.standard_normal(xyz.shape[0])
    g = op.element_gradient(u, lam)
    lam0 = np.where(mask == 1, 0.0, lam)
    go = orc.thermal_element_gradient(xyz, conn, np.exp(lnk), u, lam0)
    assert np.abs(g - go).max() <= 1e-12 * np.abs(go).max()
    xyz, conn, mask, vals, E_e = halfspace(orc, 2, 2, 2, curved=True)
    mesh, d = setup(geo, xyz, conn, mask, vals)
    op = geo.ElasticityOperator(mesh, d, geo.IsotropicElasticity(1e11, 0.25), E_e)
    u, lam = rng.standard_normal(3 * xyz.shape[0]), rng.standard_normal(3 * xyz.shape[0])
    g = op.element_gradient(u, lam)
    go = orc.elasticity_element_gradient(xyz, conn, E_e, 0.25, u, np.where(mask == 1, 0.0, lam))
    assert np.abs(g - go).max() <= 1e-12 * np.abs(go).max()


def misfit(u, obs, that):
    return 0.5 * np.sum((u[obs] - that[obs]) ** 2)


def test_thermal_vjp_vs_finite_differences_and_cpu_adjoint(orc, geo):
    xyz, conn, mask, vals, lnk, mesh, d = thermal_setup(orc, geo)
    f = orc.assemble_thermal_load(xyz, conn, 1e-6)
    tight = geo.ConjugateGradient().with_max_iterations(20000).with_tolerance(1e-13)
    op = geo.ThermalOperator(mesh, d, np.exp(lnk))
    free = np.nonzero(mask == 0)[0]
    obs = free[np.random.default_rng(4).choice(free.size, 60, replace=False)]
    u, _ = op.forward(f, tight)
    that = u + np.random.default_rng(5).normal(0, 5.0, u.size)
    dJ = np.zeros_like(u)
    dJ[obs] = u[obs] - that[obs]
    for prec in ("fp64", "mixed"):
        s = geo.ConjugateGradient().with_max_iterations(20000).with_tolerance(1e-13).with_precision(prec)
        grad, st = op.vjp(dJ, u=u, solver=s)
        assert st.converged
        grad_r, _ = op.vjp(dJ, u=None, f=f, solver=s)  # recompute-forward path
        assert np.abs(grad_r - grad).max() <= 1e-7 * np.abs(grad).max()
        # central finite differences on a few elements, FP64 solves to 1e-13
        h = 1e-6
        for e in np.random.default_rng(6).choice(conn.shape[0], 6, replace=False):
            Jp = Jm = None
            for sgn in (1, -1):
                lk = lnk.copy()
                lk[e] += sgn * h
                op.set_coefficients(np.exp(lk))
                up, _ = op.forward(f, tight)
                if sgn == 1:
                    Jp = misfit(up, obs, that)
                else:
                    Jm = misfit(up, obs, that)
            op.set_coefficients(np.exp(lnk))
            fd = (Jp - Jm) / (2 * h)
            assert abs(grad[e] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(grad).max()), (prec, e, grad[e], fd)
    # FP64 CPU adjoint from the oracle's assembled CSR
    K = orc.assemble_thermal_stiffness(xyz, conn, k_e=np.exp(lnk))
    Kb, fb = orc.apply_dirichlet_bcs(K, f, mask, vals)
    uo, _ = orc.cg_solve(Kb, fb, 20000, 1e-14)
    rhs = np.where(mask == 1, 0.0, np.where(np.isin(np.arange(u.size), obs), uo - that, 0.0))
    lam, _ = orc.cg_solve(Kb, rhs, 20000, 1e-14)
    go = orc.thermal_element_gradient(xyz, conn, np.exp(lnk), uo, lam)
    grad, _ = op.vjp(dJ, u=u, solver=tight)
    assert np.abs(grad - go).max() <= 1e-6 * np.abs(go).max()


def test_elasticity_vjp_vs_finite_differences(orc, geo):
    xyz, conn, mask, vals, E_e = halfspace(orc, 3, 3, 2)
    mesh, d = setup(geo, xyz, conn, mask, vals)
    mat = geo.IsotropicElasticity(1e11, 0.25)
    op = geo.ElasticityOperator(mesh, d, mat, E_e)
    f = orc.assemble_gravity_load(xyz, conn, 3300.0, [0, 0, -9.81])
    tight = geo.ConjugateGradient().with_max_iterations(20000).with_tolerance(1e-13)
    u, st = op.forward(f, tight)
    assert st.converged
    top = np.nonzero(np.abs(xyz[:, 2] - 50e3) < 1.0)[0]
    obs = 3 * top + 2
    that = u.copy()
    that[obs] += 1e-3 * np.random.default_rng(8).standard_normal(obs.size)
    dJ = np.zeros_like(u)
    dJ[obs] = u[obs] - that[obs]
    grad, _ = op.vjp(dJ, u=u, solver=tight)  # dJ/d(ln E_e)

    def J_at(lnE):
        op.set_coefficients(np.exp(lnE))
        up, _ = op.forward(f, tight)
        return 0.5 * np.sum((up[obs] - that[obs]) ** 2)

    # Central differences, h = 1e-6. Components far below the largest gradient
    # are dominated by where the perturbed CG solves stop (a different iteration
    # count moves J by the solve's error), so the per-element check takes
    # elements whose gradient is at least 5% of the largest; a random-direction
    # derivative covers all elements at once.
    h = 1e-6
    lnE = np.log(E_e)
    big = np.nonzero(np.abs(grad) >= 0.05 * np.abs(grad).max())[0]
    for e in np.random.default_rng(9).choice(big, min(5, big.size), replace=False):
        d = np.zeros_like(lnE)
        d[e] = h
        fd = (J_at(lnE + d) - J_at(lnE - d)) / (2 * h)
        assert abs(grad[e] - fd) <= 1e-5 * abs(fd), (e, grad[e], fd)
    d = np.random.default_rng(10).standard_normal(lnE.size)
    d /= np.linalg.norm(d)
    fd = (J_at(lnE + h * d) - J_at(lnE - h * d)) / (2 * h)
    op.set_coefficients(E_e)
    assert abs(grad @ d - fd) <= 1e-5 * abs(fd), (grad @ d, fd)
