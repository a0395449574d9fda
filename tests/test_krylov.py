"""BiCGSTAB::solve (linalg/iterative.rs:150-301) and GMRES::solve (:303-479), the
siblings of the ConjugateGradient drop-in.

CPU: the oracle's restatements on the reference's 2x2 system (iterative.rs:491-504),
against scipy's direct solution of nonsymmetric systems, and against CG on an
SPD thermal system; GMRES with a restart >= n solves an n x n system within n
steps. GPU: the device solvers against the oracle (solution, iteration count,
convergence flag) on the same systems, with and without the Jacobi
preconditioner; zero right-hand side, the iteration cap and argument errors."""
import numpy as np
import pytest

from conftest import thermal_problem


def nonsymmetric(n, seed):
    """A diagonally dominant convection-diffusion-like matrix plus a sparse random part."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    M = sp.diags([-1.3 * np.ones(n - 1), 4.0 + rng.random(n), -0.7 * np.ones(n - 1)], [-1, 0, 1]).tocsr()
    M = (M + 0.1 * sp.random(n, n, density=0.002, random_state=seed)).tocsr()
    M.sort_indices()
    return M, rng.normal(size=n)


def oracle_csr(orc, M):
    return orc.Csr(M.shape[0], M.shape[1], M.indptr.astype(np.int64), M.indices.astype(np.int64),
                   M.data.astype(np.float64))


def thermal_kbc(orc, n=4):
    xyz, conn, mask, vals = thermal_problem(n, orc)
    K = orc.assemble_thermal_stiffness(xyz, conn, k=3.0)
    f = orc.assemble_thermal_load(xyz, conn, 1e-6)
    Kbc, fbc = orc.apply_dirichlet_bcs(K, f, mask, vals)
    return Kbc, fbc


# ------------------------------------------------------------------------ CPU
def test_oracle_two_by_two(orc):
    A = oracle_csr(orc, __import__("scipy.sparse", fromlist=["csr_matrix"]).csr_matrix([[2.0, 1.0], [1.0, 2.0]]))
    for fn in (orc.bicgstab_solve, orc.gmres_solve):
        x, st = fn(A, np.array([3.0, 3.0]))
        assert np.allclose(x, 1.0, atol=1e-6) and st.converged


def test_oracle_nonsymmetric_against_direct(orc):
    import scipy.sparse.linalg as spl
    M, b = nonsymmetric(1500, 7)
    xs = spl.spsolve(M.tocsc(), b)
    A = oracle_csr(orc, M)
    for fn, kw in ((orc.bicgstab_solve, {}), (orc.gmres_solve, {}), (orc.gmres_solve, {"restart": 30}),
                   (orc.bicgstab_solve, {"use_preconditioner": False})):
        x, st = fn(A, b, max_iterations=5000, **kw)
        assert st.converged
        assert np.linalg.norm(M @ x - b) < 1e-8 * np.linalg.norm(b) * 1.0001
        assert np.linalg.norm(x - xs) < 1e-6 * np.linalg.norm(xs)


def test_oracle_spd_matches_cg_and_full_gmres(orc):
    Kbc, fbc = thermal_kbc(orc)
    xc, _ = orc.cg_solve(Kbc, fbc, max_iterations=5000, tolerance=1e-12)
    for fn in (orc.bicgstab_solve, orc.gmres_solve):
        x, st = fn(Kbc, fbc, max_iterations=5000, tolerance=1e-12)
        assert st.converged and np.linalg.norm(x - xc) < 1e-9 * np.linalg.norm(xc)
    # GMRES without restarts is exact after n steps in exact arithmetic
    M, b = nonsymmetric(40, 3)
    x, st = orc.gmres_solve(oracle_csr(orc, M), b, restart=40, tolerance=1e-12)
    assert st.converged and st.iterations <= 40


# ------------------------------------------------------------------------ GPU
def gpu_csr(geo, M):
    return geo.CsrMatrix.from_arrays(M.shape[0], M.shape[1], M.indptr, M.indices, M.data)


def oracle_to_scipy(A):
    return A.to_scipy().tocsr()


@pytest.mark.gpu
@pytest.mark.parametrize("system", ["nonsymmetric", "thermal", "two"])
@pytest.mark.parametrize("precond", [True, False])
def test_device_solvers_match_oracle(orc, geo, system, precond):
    if system == "nonsymmetric":
        M, b = nonsymmetric(3000, 11)
        A = oracle_csr(orc, M)
    elif system == "thermal":
        A, b = thermal_kbc(orc, 5)
        M = oracle_to_scipy(A)
    else:
        import scipy.sparse as sp
        M, b = sp.csr_matrix([[2.0, 1.0], [1.0, 2.0]]), np.array([3.0, 3.0])
        A = oracle_csr(orc, M)
    G = gpu_csr(geo, M)
    cases = [(geo.BiCGSTAB(), orc.bicgstab_solve, {}), (geo.GMRES(), orc.gmres_solve, {}),
             (geo.GMRES().with_restart(25), orc.gmres_solve, {"restart": 25})]
    for solver, ref, kw in cases:
        solver.with_max_iterations(5000).with_preconditioner(precond)
        x, st = solver.solve(G, b)
        xr, sr = ref(A, b, max_iterations=5000, use_preconditioner=precond, **kw)
        assert st.converged == bool(sr.converged) == True  # noqa: E712
        assert abs(st.iterations - sr.iterations) <= 2, (solver.name, st.iterations, sr.iterations)
        assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr)
        assert np.linalg.norm(M @ x - b) <= 1.0001e-8 * np.linalg.norm(b)


@pytest.mark.gpu
def test_device_solvers_edge_cases(orc, geo):
    M, b = nonsymmetric(500, 5)
    G = gpu_csr(geo, M)
    for solver in (geo.BiCGSTAB(), geo.GMRES()):
        x, st = solver.solve(G, np.zeros(500))  # iterative.rs:191-193 / :347-349
        assert st.iterations == 0 and st.converged and not np.any(x)
        x, st = solver.with_max_iterations(3).solve(G, b)  # the cap: not converged, no exception
        assert not st.converged and st.iterations == 3
    for bad in (0, 65):
        with pytest.raises(geo.GeoError):
            geo.GMRES().with_restart(bad).solve(G, b)
