"""Pins the CPU oracle against the reference's own known-answer tests (CPU only).

The reference (Rust) cannot be built here, so the oracle is anchored on every
test the reference holds for this path, restated with the same inputs and
tolerances: basis.rs:386-483, quadrature.rs:116-158, element.rs:325-386,
mechanics/element.rs:320-390, mechanics/body_force.rs:118-211,
mesh_generator_improved.rs:176-227, iterative.rs:490-504,
preconditioner.rs:212-230, direct.rs:101-143, tests/curved_element.rs:6-53,
benchmarks/shape_functions/mod.rs:26-248, and the analytic solutions of
benchmarks/thermal_1d_improved_mesh.rs:9-13 and benchmarks/elasticity_patch_test.rs:29-32.
"""
import numpy as np
import pytest

UNIT = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0],
                 [0, 0, 0.5], [0.5, 0, 0.5], [0, 0.5, 0.5]], dtype=np.float64)


def tet10_from_vertices(v):
    v = np.asarray(v, dtype=np.float64)
    e = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]
    return np.vstack([v] + [(v[a] + v[b]) * 0.5 for a, b in e])


# ----------------------------------------------------------------- basis.rs:386-483
def test_partition_of_unity(orc):
    for L in ([0.25] * 4, [1, 0, 0, 0], [0, 1, 0, 0], [0.5, 0.5, 0, 0], [0.1, 0.2, 0.3, 0.4],
              [0.7, 0.1, 0.1, 0.1], [0.0, 0.33, 0.33, 0.34]):
        assert abs(orc.shape_functions(L).sum() - 1.0) <= 1e-14


def test_kronecker_delta(orc):
    nodes_L = [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1], [0.5, 0.5, 0, 0], [0, 0.5, 0.5, 0],
               [0.5, 0, 0.5, 0], [0.5, 0, 0, 0.5], [0, 0.5, 0, 0.5], [0, 0, 0.5, 0.5]]
    for i, L in enumerate(nodes_L):
        N = orc.shape_functions(L)
        expect = np.zeros(10)
        expect[i] = 1.0
        assert np.abs(N - expect).max() <= 1e-14


def test_reference_volume(orc):
    assert abs(orc.element_volume(UNIT) - 1.0 / 6.0) <= 1e-14
    # shape_functions/mod.rs:200-248
    assert abs(orc.element_volume(tet10_from_vertices([[0, 0, 0], [2, 0, 0], [0, 2, 0], [0, 0, 2]])) - 8.0 / 6.0) <= 1e-14


def test_derivative_sum_and_linear_field(orc):
    # shape_functions/mod.rs:150-198 (sum of Cartesian derivatives = 0)
    for L in ([0.25] * 4, [0.1, 0.2, 0.3, 0.4]):
        d = orc.shape_derivatives_cartesian(L, UNIT)
        assert np.abs(d.sum(axis=0)).max() <= 1e-12
    # linear field reproduction (mod.rs:94-148): interpolate f = 2x + 3y + 4z + 5
    f = lambda p: 2 * p[..., 0] + 3 * p[..., 1] + 4 * p[..., 2] + 5
    vals = f(UNIT)
    for p in ([0.25, 0.25, 0.25], [0.1, 0.2, 0.3], [0.4, 0.3, 0.2], [0.6, 0.2, 0.1]):
        L = [1 - sum(p), *p]
        assert abs(orc.shape_functions(L) @ vals - f(np.array(p))) <= 1e-12


# ----------------------------------------------------------------- quadrature.rs:116-158
def test_quadrature_rules(orc):
    for rule in (1, 4, 5, 11):
        pts, w = orc.quadrature(rule)
        assert abs(w.sum() - 1.0 / 6.0) <= 1e-14
        assert np.abs(pts.sum(axis=1) - 1.0).max() <= 1e-14
    pts, w = orc.quadrature(4)
    assert abs((pts[:, 1] ** 2 * w).sum() - 1.0 / 60.0) <= 1e-14


# ----------------------------------------------------------------- element.rs:325-386
def test_thermal_element_properties(orc):
    K = orc.thermal_stiffness(UNIT, 1.0)
    assert np.abs(K - K.T).max() <= 1e-14
    assert (np.diag(K) > 0).all()
    assert np.abs(K.sum(axis=1)).max() <= 1e-12
    M = orc.thermal_mass(UNIT, 1.0, 1.0)
    assert np.abs(M - M.T).max() <= 1e-14
    f = orc.thermal_load(UNIT, 6.0)
    assert abs(f.sum() - 6.0 * orc.element_volume(UNIT)) <= 1e-12


# ----------------------------------------------------------------- curved_element.rs:6-53
def test_curved_element_volume(orc):
    nodes = UNIT.copy()
    pts, w = orc.quadrature(4)
    vs = sum(wi * abs(orc.det3(orc.jacobian(L, nodes))) for L, wi in zip(pts, w))
    assert abs(vs - 1.0 / 6.0) <= 1e-10
    nodes[4, 1] -= 0.1
    vc = sum(wi * abs(orc.det3(orc.jacobian(L, nodes))) for L, wi in zip(pts, w))
    assert vc > vs
    assert abs(orc.shape_functions([0.25] * 4).sum() - 1.0) <= 1e-10


# ----------------------------------------------------------------- mechanics
def test_elasticity_element(orc):
    # mechanics/element.rs:320-390
    K = orc.elasticity_stiffness(UNIT, 100e9, 0.25)
    assert np.allclose(K, K.T, rtol=1e-12, atol=1e-6)
    ev = np.sort(np.linalg.eigvalsh(0.5 * (K + K.T)))
    assert (np.abs(ev[:6]) < 1e3).all()
    assert (ev[6:] > 1e6).all()
    K2 = orc.elasticity_stiffness(UNIT, 200e9, 0.25)
    assert np.abs(K2 - 2 * K).max() <= 1e-6
    # constitutive.rs:63-102
    D = orc.constitutive_matrix(100e9, 0.25)
    lam = 100e9 * 0.25 / (1.25 * 0.5)
    mu = 100e9 / 2.5
    assert D[0, 0] == pytest.approx(lam + 2 * mu, rel=1e-14)
    assert D[0, 1] == pytest.approx(lam, rel=1e-14)
    assert D[3, 3] == pytest.approx(mu, rel=1e-14)


def test_gravity_load(orc):
    # body_force.rs:118-211
    f = orc.gravity_load(UNIT, 3000.0, [0, 0, -9.81])
    V = orc.element_volume(UNIT)
    assert f[2::3].sum() == pytest.approx(-3000.0 * V * 9.81, abs=1e-6)
    assert (np.abs(f[2::3]) > 1e-10).all()
    fx = orc.gravity_load(UNIT, 3000.0, [9.81, 0, 0])
    assert fx[0::3].sum() == pytest.approx(3000.0 * V * 9.81, abs=1e-6)
    assert abs(fx[1::3].sum()) <= 1e-10 and abs(fx[2::3].sum()) <= 1e-10
    assert np.abs(orc.gravity_load(UNIT, 3000.0, [0, 0, 0])).max() <= 1e-12


# ----------------------------------------------------------------- mesh_generator_improved.rs:176-227
def test_mesh_generator(orc):
    xyz, conn = orc.generate_cube(1, 1, 1, 1.0, 1.0, 1.0)
    assert conn.shape[0] == 6
    xyz2, conn2 = orc.generate_cube(2, 2, 2, 1.0, 1.0, 1.0)
    assert conn2.shape[0] == 48
    keys = {tuple(np.round(p * 1000).astype(np.int64)) for p in xyz2}
    assert len(keys) == xyz2.shape[0]
    for el in conn:
        z = np.unique(np.round(xyz[el[:4], 2], 10))
        assert z.size >= 2
    # the v2<->v3 swap leaves every element positively oriented
    for el in conn2:
        v = xyz2[el[:4]]
        assert np.linalg.det(np.stack([v[1] - v[0], v[2] - v[0], v[3] - v[0]])) > 0


# ----------------------------------------------------------------- linalg tests
def test_cg_2x2_and_jacobi_and_lu(orc):
    A = orc.csr_from_triplets(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [2.0, 1.0, 1.0, 2.0])
    x, st = orc.cg_solve(A, [3.0, 3.0])
    assert np.abs(x - 1.0).max() <= 1e-6 and st.converged
    x, st = orc.lu_solve(A, [3.0, 3.0])
    assert np.abs(x - 1.0).max() <= 1e-10 and st.converged and st.relative_residual < 1e-8
    D = orc.csr_from_triplets(10, 10, range(10), range(10), np.arange(1, 11, dtype=float))
    x, st = orc.lu_solve(D, np.arange(1, 11, dtype=float) ** 2)
    assert np.abs(x - np.arange(1, 11)).max() <= 1e-10
    # Jacobi on a diagonal matrix converges in one CG iteration (preconditioner.rs:212-230)
    D3 = orc.csr_from_triplets(3, 3, [0, 1, 2], [0, 1, 2], [2.0, 4.0, 8.0])
    x, st = orc.cg_solve(D3, [2.0, 4.0, 8.0])
    assert np.abs(x - 1.0).max() <= 1e-14 and st.iterations == 0


def test_sprs_merge_semantics(orc):
    # duplicates summed, columns sorted, explicit zeros kept
    A = orc.csr_from_triplets(2, 3, [1, 0, 1, 0, 0], [2, 1, 0, 1, 0], [1.0, 2.0, 3.0, -2.0, 5.0])
    assert A.indptr.tolist() == [0, 2, 4]
    assert A.indices.tolist() == [0, 1, 0, 2]
    assert A.data.tolist() == [5.0, 0.0, 3.0, 1.0]


# ----------------------------------------------------------------- analytic solutions
def test_thermal_analytic_profile(orc):
    """thermal_1d_improved_mesh.rs:9-13, exact for P2 up to the solver tolerance."""
    for n in (2, 4):
        xyz, conn = orc.generate_cube(n, n, n, 1000.0, 1000.0, 600.0)
        mask, vals = orc.thermal_bc(xyz, 600.0)
        K = orc.assemble_thermal_stiffness(xyz, conn, 3.0)
        f = orc.assemble_thermal_load(xyz, conn, 1e-6)
        Kb, fb = orc.apply_dirichlet_bcs(K, f, mask, vals)
        x, st = orc.cg_solve(Kb, fb, 1000, 1e-12)
        z = xyz[:, 2]
        ta = 1280.0 - 1280.0 * z / 600.0 + 1e-6 / 6.0 * z * (600.0 - z)
        assert st.converged and np.abs(x - ta).max() < 1e-5


def test_elasticity_patch_test(orc):
    """elasticity_patch_test.rs:14-107: constant-strain field reproduced exactly."""
    L_ = 10e3
    E, nu, s0 = 100e9, 0.25, 10e6
    ezz, exx = s0 / E, -nu * s0 / E
    xyz, conn = orc.generate_cube(2, 2, 2, L_, L_, L_)
    n = xyz.shape[0]
    mask = np.zeros(3 * n, np.uint8)
    vals = np.zeros(3 * n)
    for i, (x, y, z) in enumerate(xyz):
        if abs(z) < 1.0 or abs(z - L_) < 1.0:
            mask[3 * i + 2], vals[3 * i + 2] = 1, ezz * z
        if abs(x) < 1.0:
            mask[3 * i], vals[3 * i] = 1, exx * x
        if abs(y) < 1.0:
            mask[3 * i + 1], vals[3 * i + 1] = 1, exx * y
    K = orc.assemble_elasticity_stiffness(xyz, conn, E, nu)
    Kb, fb = orc.apply_dirichlet_bcs(K, np.zeros(3 * n), mask, vals)
    u, st = orc.cg_solve(Kb, fb, 5000, 1e-12)
    assert st.converged
    exact = np.stack([exx * xyz[:, 0], exx * xyz[:, 1], ezz * xyz[:, 2]], axis=1).ravel()
    assert np.abs(u - exact).max() <= 1e-6 * np.abs(exact).max()


def test_survey_structure_counts(orc):
    """nnz of config 1 (6^3): K 54,793 and K_bc 44,513; CG iterations 58 / 74."""
    xyz, conn = orc.generate_cube(6, 6, 6, 1000.0, 1000.0, 600.0)
    mask, vals = orc.thermal_bc(xyz, 600.0)
    K = orc.assemble_thermal_stiffness(xyz, conn, 3.0)
    Kb, fb = orc.apply_dirichlet_bcs(K, orc.assemble_thermal_load(xyz, conn, 1e-6), mask, vals)
    assert (K.nnz, Kb.nnz) == (54793, 44513)
    assert orc.cg_solve(Kb, fb, 1000, 1e-8)[1].iterations == 58
    assert orc.cg_solve(Kb, fb, 1000, 1e-10)[1].iterations == 74


def test_serial_and_parallel_assembly_agree(orc):
    """assembly.rs:1048-1070 (nnz equal; here the values are compared too)."""
    xyz, conn = orc.generate_cube(3, 3, 3, 1.0, 1.0, 1.0)
    a = orc.assemble_thermal_stiffness(xyz, conn, 1.0, parallel=False)
    b = orc.assemble_thermal_stiffness(xyz, conn, 1.0, parallel=True)
    assert a.nnz == b.nnz and np.array_equal(a.indices, b.indices) and np.array_equal(a.data, b.data)
