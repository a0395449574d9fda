"""DirectSolver::solve (linalg/direct.rs:28-73): dense LU with partial pivoting.

CPU: the oracle's restatement on the reference's own known-answer test (the
2x2 system [2 1; 1 2] x = [3; 3], x = [1; 1], direct.rs:103-122), against
scipy's sparse LU on nonsymmetric, SPD thermal and pivot-forcing systems, and
its singular-matrix failure; the Python mirror's fixed tolerances and its
refusal of a matrix-free operator (direct.rs:75-95).
GPU: the device solve against the oracle (solution, residual, flags) on the
same systems and on sizes that take each work split of the kernel (several
warps per row, one warp per row, more rows than warps); pivot ties; singular
matrices (at the first column and in the middle of the elimination) raise
GEO_ERR_SINGULAR_MATRIX and leave the context usable; argument errors."""
import numpy as np
import pytest

from conftest import thermal_problem


def oracle_csr(orc, M):
    return orc.Csr(M.shape[0], M.shape[1], M.indptr.astype(np.int64), M.indices.astype(np.int64),
                   M.data.astype(np.float64))


def csr(rows):
    import scipy.sparse as sp
    M = sp.csr_matrix(np.asarray(rows, dtype=np.float64))
    M.sort_indices()
    return M


def nonsymmetric(n, seed, density=0.01):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    M = sp.diags([-1.3 * np.ones(n - 1), 4.0 + rng.random(n), -0.7 * np.ones(n - 1)], [-1, 0, 1]).tocsr()
    if density:
        M = (M + 0.1 * sp.random(n, n, density=density, random_state=seed)).tocsr()
    M.sort_indices()
    return M, rng.normal(size=n)


def dense_random(n, seed):
    """A dense matrix with no diagonal dominance: pivoting happens at most columns."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    M = sp.csr_matrix(rng.normal(size=(n, n)))
    M.sort_indices()
    return M, rng.normal(size=n)


def thermal_kbc(orc, n=4):
    xyz, conn, mask, vals = thermal_problem(n, orc)
    K = orc.assemble_thermal_stiffness(xyz, conn, k=3.0)
    f = orc.assemble_thermal_load(xyz, conn, 1e-6)
    return orc.apply_dirichlet_bcs(K, f, mask, vals)


def pivot_forcing(n):
    """Zero diagonal (a cyclic shift plus a small perturbation): every column pivots."""
    import scipy.sparse as sp
    P = sp.eye(n, k=1, format="csr") + sp.eye(n, k=-(n - 1), format="csr")
    M = (P * 2.0 + 0.25 * sp.eye(n, k=-1, format="csr")).tocsr()
    M.sort_indices()
    return M, np.arange(1.0, n + 1.0)


# ------------------------------------------------------------------------ CPU
def test_oracle_reference_known_answer(orc):
    x, st = orc.lu_solve(oracle_csr(orc, csr([[2.0, 1.0], [1.0, 2.0]])), np.array([3.0, 3.0]))
    assert abs(x[0] - 1.0) <= 1e-10 and abs(x[1] - 1.0) <= 1e-10  # direct.rs:118-119
    assert st.converged and st.relative_residual < 1e-8 and st.iterations == 0


def test_oracle_against_scipy(orc):
    import scipy.sparse.linalg as spl
    systems = [nonsymmetric(400, 3), pivot_forcing(50), dense_random(120, 5)]
    Kbc, fbc = thermal_kbc(orc)
    systems.append((Kbc.to_scipy().tocsr(), fbc))
    for M, b in systems:
        x, st = orc.lu_solve(oracle_csr(orc, M), b)
        xs = spl.spsolve(M.tocsc(), b)
        assert np.linalg.norm(x - xs) <= 1e-9 * np.linalg.norm(xs)
        assert st.converged and st.residual_norm == pytest.approx(np.linalg.norm(M @ x - b), rel=1e-6, abs=1e-300)


def test_oracle_singular(orc):
    for rows in ([[1.0, 2.0], [2.0, 4.0]], [[1.0, 1.0, 0.0], [1.0, 1.0, 0.0], [0.0, 0.0, 1.0]]):
        with pytest.raises(np.linalg.LinAlgError):
            orc.lu_solve(oracle_csr(orc, csr(rows)), np.ones(len(rows)))


def test_mirror_fixed_tolerances_and_operator_refusal():
    import geo_simulator_b200 as geo
    s = geo.DirectSolver.new()
    assert s.name == "Direct (Sparse LU)"
    s.set_tolerance(1e-3)
    s.set_abs_tolerance(1e-3)
    assert s.tolerance() == 0.0 and s.abs_tolerance() == 0.0  # direct.rs:92-95
    with pytest.raises(geo.GeoError, match="does not support matrix-free"):
        s.solve_with_operator(None, np.ones(3))


# ------------------------------------------------------------------------ GPU
def gpu_csr(geo, M):
    return geo.CsrMatrix.from_arrays(M.shape[0], M.shape[1], M.indptr, M.indices, M.data)


@pytest.mark.gpu
def test_device_reference_known_answer(geo):
    x, st = geo.DirectSolver().solve(gpu_csr(geo, csr([[2.0, 1.0], [1.0, 2.0]])), np.array([3.0, 3.0]))
    assert abs(x[0] - 1.0) <= 1e-10 and abs(x[1] - 1.0) <= 1e-10
    assert st.converged and st.relative_residual < 1e-8 and st.iterations == 0


@pytest.mark.gpu
@pytest.mark.parametrize("system", ["nonsymmetric_60", "nonsymmetric_500", "thermal", "pivot_forcing",
                                    "dense_300", "dense_1200", "nonsymmetric_2500", "banded_5000", "one", "ties"])
def test_device_matches_oracle(orc, geo, system):
    if system.startswith("nonsymmetric"):
        M, b = nonsymmetric(int(system.split("_")[1]), 11)
    elif system.startswith("banded"):  # no fill-in: more rows than warps for most columns
        M, b = nonsymmetric(int(system.split("_")[1]), 17, density=0)
    elif system.startswith("dense"):
        M, b = dense_random(int(system.split("_")[1]), 13)
    elif system == "thermal":
        A, b = thermal_kbc(orc, 5)
        M = A.to_scipy().tocsr()
    elif system == "pivot_forcing":
        M, b = pivot_forcing(257)
    elif system == "one":
        M, b = csr([[-4.0]]), np.array([2.0])
    else:  # equal |a_ik| in a column: the first row is the pivot
        M, b = csr([[1.0, 2.0, 0.5], [-1.0, 3.0, 1.0], [1.0, -1.0, 2.0]]), np.array([1.0, 2.0, 3.0])
    xr, sr = orc.lu_solve(oracle_csr(orc, M), b)
    x, st = geo.DirectSolver().solve(gpu_csr(geo, M), b)
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)
    assert st.iterations == 0 and st.converged == bool(sr.converged) == True  # noqa: E712
    r = np.linalg.norm(M @ x - b)
    assert st.residual_norm == pytest.approx(r, rel=1e-6, abs=1e-12 * np.linalg.norm(b))
    assert st.relative_residual == pytest.approx(st.residual_norm / np.linalg.norm(b), rel=1e-12)


@pytest.mark.gpu
def test_device_zero_rhs_and_device_buffers(geo):
    import torch
    M, b = nonsymmetric(300, 2)
    A = gpu_csr(geo, M)
    x, st = geo.DirectSolver().solve(A, np.zeros(300))
    assert not np.any(x) and st.residual_norm == 0.0 and st.converged  # ||b|| < 1e-14: rel = ||r||
    bd = torch.tensor(b, device="cuda")
    xd, _ = geo.DirectSolver().solve(A, bd)
    xh, _ = geo.DirectSolver().solve(A, b)
    assert np.array_equal(xd.cpu().numpy(), xh)


@pytest.mark.gpu
def test_device_singular_and_arguments(geo):
    s = geo.DirectSolver()
    for rows in ([[1.0, 2.0], [2.0, 4.0]], [[1.0, 1.0, 0.0], [1.0, 1.0, 0.0], [0.0, 0.0, 1.0]],
                 [[0.0, 0.0], [0.0, 0.0]]):
        with pytest.raises(geo.GeoError, match="GEO_ERR_SINGULAR_MATRIX"):
            s.solve(gpu_csr(geo, csr(rows)), np.ones(len(rows)))
    x, st = s.solve(gpu_csr(geo, csr([[2.0, 1.0], [1.0, 2.0]])), np.array([3.0, 3.0]))  # still usable
    assert np.allclose(x, 1.0) and st.converged
    import scipy.sparse as sp
    with pytest.raises(geo.GeoError, match="GEO_ERR_INVALID_ARG"):
        s.solve(gpu_csr(geo, sp.eye(16385, format="csr")), np.ones(16385))
