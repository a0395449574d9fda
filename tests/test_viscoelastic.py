"""Maxwell viscoelasticity: MaxwellViscoelasticity (mechanics/constitutive.rs:286-395),
the history force of assemble_maxwell_viscoelastic_parallel (assembly.rs:959-1020,
mechanics/element.rs:257-296), update_stresses_maxwell (mechanics/stress_update.rs:
39-143) and BackwardEuler (fem/time_integration.rs:38-160).

CPU: the oracle and the Python mirror against the reference's own tests and the
identity f_history(D eps) = -K u for a constant-strain field.
GPU: history force, stress update and the assembled system against the oracle,
and the stress-relaxation benchmark (maxwell_stress_relaxation.rs) against its
discrete decay, through the CSR step and the matrix-free step."""
import numpy as np
import pytest

E, NU, MU = 100e9, 0.25, 1e19


def linear_field(xyz, eps):
    """u = eps . x for a symmetric strain tensor eps (3x3)."""
    return (xyz @ np.asarray(eps).T).ravel()


def voigt(eps):
    return np.array([eps[0, 0], eps[1, 1], eps[2, 2], 2 * eps[0, 1], 2 * eps[1, 2], 2 * eps[0, 2]])


EPS = np.array([[1e-3, 2e-4, -1e-4], [2e-4, -5e-4, 3e-4], [-1e-4, 3e-4, 7e-4]])


# ------------------------------------------------------------------------ CPU
def test_material_pins(geo, orc):
    """constitutive.rs:595-730."""
    m = geo.MaxwellViscoelasticity.new(E, NU, MU)
    assert m.shear_modulus() == pytest.approx(E / (2 * (1 + NU)))
    assert m.relaxation_time() == pytest.approx(MU / m.shear_modulus())
    D = m.elastic_matrix()
    assert np.allclose(D, orc.constitutive_matrix(E, NU), rtol=1e-14, atol=0)
    assert np.allclose(m.effective_constitutive_matrix(1e-20), D, rtol=1e-12)
    assert np.abs(m.effective_constitutive_matrix(1e6 * m.relaxation_time())).max() < 0.01 * D[0, 0]
    assert np.allclose(m.effective_constitutive_matrix(m.relaxation_time()), D / 2, rtol=1e-14)
    for bad in ((-1.0, NU, MU), (E, 0.5, MU), (E, NU, 0.0)):
        with pytest.raises(geo.GeoError):
            geo.MaxwellViscoelasticity.new(*bad)


def test_oracle_stress_update_pins(orc):
    """stress_update.rs:154-246 (zero displacement, dimensions, relaxation to 2/3)."""
    xyz, conn = orc.generate_cube(1, 1, 1, 1.0, 1.0, 1.0)
    G = E / (2 * (1 + NU))
    tau = MU / G
    n = 3 * xyz.shape[0]
    zero = orc.update_stresses_maxwell(xyz, conn, E, NU, MU, np.zeros(n), np.zeros(n), 1.0, np.zeros((6, 6)))
    assert zero.shape == (6, 6) and np.abs(zero).max() == 0.0
    s0 = np.zeros((6, 6))
    s0[0, 0] = 1e6
    u = np.full(n, 0.01)
    s1 = orc.update_stresses_maxwell(xyz, conn, E, NU, MU, u, u, tau, s0)
    assert abs(s1[0, 0] - 1e6 * 2 / 3) / (1e6 * 2 / 3) < 1e-6


def test_oracle_history_force_is_minus_k_u(orc):
    """For u = eps x (constant strain), sigma = D eps on every element and
    -sum B^T sigma = -K u, so f_history = -K u on every node."""
    xyz, conn = orc.generate_cube(2, 2, 2, 1.0, 1.2, 0.8)
    D = orc.constitutive_matrix(E, NU)
    sig = np.tile(D @ voigt(EPS), (conn.shape[0], 1))
    f = orc.maxwell_history_force(xyz, conn, sig)
    K = orc.assemble_elasticity_stiffness(xyz, conn, E=E, nu=NU)
    ku = orc.csr_apply(K, linear_field(xyz, EPS))
    assert np.abs(f + ku).max() <= 1e-9 * np.abs(ku).max()


def test_backward_euler_host_logic(geo):
    """time_integration.rs:164-222."""
    be = geo.BackwardEuler.new(30, 0.5)
    assert be.current_time() == 0.0 and be.current_displacement().shape == (30,)
    be.time, be.displacement[:] = 2.0, 1.0
    be.reset()
    assert be.current_time() == 0.0 and not be.current_displacement().any()
    be.set_timestep(0.25)
    assert be.dt == 0.25
    for bad in ((30, -1.0), (0, 1.0)):
        with pytest.raises(geo.GeoError):
            geo.BackwardEuler.new(*bad)
    with pytest.raises(geo.GeoError):
        be.set_timestep(-1.0)


# ------------------------------------------------------------------------ GPU
def curved_mesh(orc, n=2, seed=4):
    xyz, conn = orc.generate_cube(n, n, n, 1.0, 1.0, 1.0)
    nv = (n + 1) ** 3
    xyz = xyz.copy()
    xyz[nv:] += np.random.default_rng(seed).uniform(-0.02, 0.02, (xyz.shape[0] - nv, 3)) / n
    return xyz, conn


@pytest.mark.gpu
def test_history_force_and_stress_update_match_oracle(orc, geo):
    xyz, conn = curved_mesh(orc)
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    rng = np.random.default_rng(5)
    sig = rng.normal(0, 1e6, (conn.shape[0], 6))
    f = geo.Assembler.maxwell_history_force(mesh, sig)
    fo = orc.maxwell_history_force(xyz, conn, sig)
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()
    u0, u1 = rng.normal(0, 1e-3, (2, 3 * xyz.shape[0]))
    mesh.stress_history = geo.StressHistory(conn.shape[0])
    mesh.stress_history.update_all(sig)
    m = geo.MaxwellViscoelasticity.new(E, NU, MU)
    d = geo.DofManager(xyz.shape[0], 3)
    for dt in (0.0, 0.3 * m.relaxation_time(), 5 * m.relaxation_time()):
        s = geo.update_stresses_maxwell(mesh, d, m, u0, u1, dt)
        so = orc.update_stresses_maxwell(xyz, conn, E, NU, MU, u0, u1, dt, sig)
        assert np.abs(s - so).max() <= 1e-12 * np.abs(so).max()


@pytest.mark.gpu
def test_assembled_maxwell_system(orc, geo):
    from test_golden import row_err
    xyz, conn = curved_mesh(orc, seed=6)
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    mesh.stress_history = geo.StressHistory(conn.shape[0])
    mesh.stress_history.update_all(np.random.default_rng(7).normal(0, 1e6, (conn.shape[0], 6)))
    d = geo.DofManager(xyz.shape[0], 3)
    m = geo.MaxwellViscoelasticity.new(E, NU, MU)
    K, fh = geo.Assembler.assemble_maxwell_viscoelastic_parallel(mesh, d, m, 0.1 * m.relaxation_time())
    Ko = orc.assemble_elasticity_stiffness(xyz, conn, E=E, nu=NU)
    ip, ix, data = K.to_host()
    assert np.array_equal(ip, Ko.indptr) and np.array_equal(ix.astype(np.int64), Ko.indices)
    assert row_err(data, Ko.data, ip) <= 1e-12
    fo = orc.maxwell_history_force(xyz, conn, mesh.stress_history.stress)
    assert np.abs(fh - fo).max() <= 1e-12 * np.abs(fo).max()
    with pytest.raises(geo.GeoError):
        geo.Assembler.assemble_maxwell_viscoelastic_parallel(mesh, geo.DofManager(xyz.shape[0], 1), m, 1.0)


@pytest.mark.gpu
def test_stress_relaxation_benchmark(geo):
    """maxwell_stress_relaxation.rs: exact uniaxial-stress displacements on every
    boundary node, elastic start, then held: the deviatoric stress decays by
    1 / (1 + dt / tau_M) per step and the pressure stays."""
    n, eps0, steps = 3, 1e-3, 6
    m = geo.MaxwellViscoelasticity.new(E, NU, MU)
    tau = m.relaxation_time()
    dt = 0.25 * tau
    mesh = geo.ImprovedMeshGenerator.generate_cube(n, n, n, 1.0, 1.0, 1.0)
    x, y, z = mesh.nodes.T
    d = geo.DofManager(mesh.num_nodes(), 3)
    bnd = (np.minimum.reduce([x, 1 - x, y, 1 - y, z, 1 - z]) < 1e-6)
    for i in np.nonzero(bnd)[0]:
        d.set_dirichlet(d.global_dof(i, 0), -NU * eps0 * x[i])
        d.set_dirichlet(d.global_dof(i, 1), -NU * eps0 * y[i])
        d.set_dirichlet(d.global_dof(i, 2), eps0 * z[i])
    mesh.stress_history = geo.StressHistory(mesh.num_elements())
    cg = geo.ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-12)
    K, _ = geo.Assembler.assemble_maxwell_viscoelastic_parallel(mesh, d, m, 1e-20)
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, np.zeros(d.total_dofs()), d)
    u0, st = cg.solve(Kb, fb)
    assert st.converged
    s0 = geo.update_stresses_maxwell(mesh, d, m, np.zeros_like(u0), u0, 1e-20)
    sigma0 = E * eps0
    assert np.allclose(s0[:, 2], sigma0, rtol=1e-6) and np.abs(s0[:, [0, 1, 3, 4, 5]]).max() < 1e-6 * sigma0
    op = geo.ElasticityOperator(mesh, d, geo.IsotropicElasticity(E, NU))
    for mode in ("csr", "operator"):
        mesh.stress_history.update_all(s0)
        be = geo.BackwardEuler.new(d.total_dofs(), dt)
        u_prev = u0
        for k in range(1, steps + 1):
            if mode == "csr":
                u, ts = be.step(mesh, d, m, np.zeros(d.total_dofs()), cg)
            else:
                u, ts = be.step_operator(op, mesh, np.zeros(d.total_dofs()), cg)
            mesh.stress_history.update_all(geo.update_stresses_maxwell(mesh, d, m, u_prev, u, dt))
            u_prev = u
            decay = (1.0 + dt / tau) ** -k
            s = mesh.stress_history.stress
            p = sigma0 / 3
            assert np.allclose(s[:, 2], p + 2 * p * decay, rtol=1e-6), (mode, k)
            assert np.allclose(s[:, 0], p - p * decay, rtol=1e-6, atol=1e-6 * sigma0), (mode, k)
        assert be.current_time() == pytest.approx(steps * dt)
