"""3-DOF elasticity on the GPU vs the oracle (assembly.rs:389-437, :906-937,
mechanics/*), plus the analytic patch test (elasticity_patch_test.rs)."""
import numpy as np
import pytest

from test_golden import row_err

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def halfspace(orc, nx, ny, nz, lx=100e3, ly=100e3, lz=50e3, curved=False, seed=5):
    xyz, conn = orc.generate_cube(nx, ny, nz, lx, ly, lz)
    rng = np.random.default_rng(seed)
    if curved:
        xyz = xyz.copy()
        nv = (nx + 1) * (ny + 1) * (nz + 1)
        xyz[nv:] += rng.uniform(-0.03, 0.03, (xyz.shape[0] - nv, 3)) * np.array([lx / nx, ly / ny, lz / nz])
    n = xyz.shape[0]
    mask = np.zeros(3 * n, np.uint8)
    for i, (x, y, z) in enumerate(xyz):
        if abs(z) < 1.0:
            mask[3 * i + 2] = 1
            if abs(x) < 1.0 and abs(y) < 1.0:
                mask[3 * i] = mask[3 * i + 1] = 1
        if abs(x) < 1.0 or abs(x - lx) < 1.0:
            mask[3 * i] = 1
        if abs(y) < 1.0 or abs(y - ly) < 1.0:
            mask[3 * i + 1] = 1
    E_e = np.exp(np.log(1e11) + 0.3 * rng.standard_normal(conn.shape[0]))
    return xyz, conn, mask, np.zeros(3 * n), E_e


def setup(geo, xyz, conn, mask, vals):
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    d = geo.DofManager(xyz.shape[0], 3)
    idx = np.nonzero(mask)[0]
    d.set_dirichlet(idx, vals[idx])
    return mesh, d


def test_element_and_assembly(orc, geo):
    xyz, conn, mask, vals, E_e = halfspace(orc, 3, 2, 2, curved=True)
    mesh, d = setup(geo, xyz, conn, mask, vals)
    mat = geo.IsotropicElasticity(1e11, 0.25)
    Ke = geo.ElasticityElement.stiffness_matrix(mesh, mat, E_e)
    for e in range(conn.shape[0]):
        ko = orc.elasticity_stiffness(xyz[conn[e]], E_e[e], 0.25)
        assert np.abs(Ke[e] - ko).max() <= 1e-12 * np.abs(ko).max()
    K = geo.Assembler.assemble_elasticity_stiffness_parallel(mesh, d, mat, E_e)
    Ko = orc.assemble_elasticity_stiffness(xyz, conn, E_e=E_e, nu=0.25)
    ip, ix, data = K.to_host()
    assert np.array_equal(ip, Ko.indptr) and np.array_equal(ix.astype(np.int64), Ko.indices)
    assert row_err(data, Ko.data, ip) <= 1e-12
    f = geo.Assembler.assemble_gravity_load(mesh, d, 3300.0, [0, 0, -9.81])
    fo = orc.assemble_gravity_load(xyz, conn, 3300.0, [0, 0, -9.81])
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, f, d)
    Kbo, fbo = orc.apply_dirichlet_bcs(Ko, fo, mask, vals)
    ip, ix, data = Kb.to_host()
    assert np.array_equal(ip, Kbo.indptr) and np.array_equal(ix.astype(np.int64), Kbo.indices)
    assert row_err(data, Kbo.data, ip) <= 1e-12
    assert np.abs(fb - fbo).max() <= 1e-12 * np.abs(fbo).max()
    u, st = geo.ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-10).solve(Kb, fb)
    uo, so = orc.cg_solve(Kbo, fbo, 5000, 1e-10)
    assert st.converged and abs(st.iterations - so.iterations) <= 2
    ul, _ = orc.lu_solve(Kbo, fbo)
    assert rel(u, ul) <= 1e-8


def test_matfree_operator(orc, geo):
    xyz, conn, mask, vals, E_e = halfspace(orc, 3, 3, 2, curved=False)
    mesh, d = setup(geo, xyz, conn, mask, vals)
    mat = geo.IsotropicElasticity(1e11, 0.25)
    Ko = orc.assemble_elasticity_stiffness(xyz, conn, E_e=E_e, nu=0.25)
    fo = orc.assemble_gravity_load(xyz, conn, 3300.0, [0, 0, -9.81])
    Kbo, fbo = orc.apply_dirichlet_bcs(Ko, fo, mask, vals)
    op = geo.ElasticityOperator(mesh, d, mat, E_e)
    assert op.char_diag == pytest.approx(orc.char_diag(Ko), rel=1e-12)
    x = np.random.default_rng(1).standard_normal(3 * xyz.shape[0])
    y_ref = orc.csr_apply(Kbo, x)
    assert rel(op.apply(x), y_ref) <= 1e-12
    assert rel(op.apply(x, precision="mixed"), y_ref) <= 1e-5
    assert np.abs(op.lift_rhs(fo) - fbo).max() <= 1e-12 * np.abs(fbo).max()
    Kd = Kbo.to_scipy().diagonal()
    assert np.abs(op.diagonal() - Kd).max() <= 1e-12 * np.abs(Kd).max()
    ul, _ = orc.lu_solve(Kbo, fbo)
    for prec in ("fp64", "mixed"):
        u, st = op.solve(fbo, geo.ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-10)
                         .with_precision(prec))
        assert st.converged and rel(u, ul) <= 1e-8, (prec, st)


def test_matfree_curved(orc, geo):
    xyz, conn, mask, vals, E_e = halfspace(orc, 2, 2, 2, curved=True)
    mesh, d = setup(geo, xyz, conn, mask, vals)
    op = geo.ElasticityOperator(mesh, d, geo.IsotropicElasticity(1e11, 0.3), E_e)
    Ko = orc.assemble_elasticity_stiffness(xyz, conn, E_e=E_e, nu=0.3)
    Kbo, _ = orc.apply_dirichlet_bcs(Ko, np.zeros(3 * xyz.shape[0]), mask, vals)
    x = np.random.default_rng(2).standard_normal(3 * xyz.shape[0])
    assert rel(op.apply(x), orc.csr_apply(Kbo, x)) <= 1e-12


def test_patch_test_exact(orc, geo):
    """elasticity_patch_test.rs:14-107 on the GPU: CSR drop-in and matrix-free."""
    L_ = 10e3
    E, nu, s0 = 100e9, 0.25, 10e6
    ezz, exx = s0 / E, -nu * s0 / E
    mesh = geo.ImprovedMeshGenerator.generate_cube(3, 3, 3, L_, L_, L_)
    xyz = mesh.nodes
    d = geo.DofManager(mesh.num_nodes(), 3)
    for i, (x, y, z) in enumerate(xyz):
        if abs(z) < 1.0 or abs(z - L_) < 1.0:
            d.set_dirichlet(d.global_dof(i, 2), ezz * z)
        if abs(x) < 1.0:
            d.set_dirichlet(d.global_dof(i, 0), exx * x)
        if abs(y) < 1.0:
            d.set_dirichlet(d.global_dof(i, 1), exx * y)
    mat = geo.IsotropicElasticity(E, nu)
    K = geo.Assembler.assemble_elasticity_stiffness_parallel(mesh, d, mat)
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, np.zeros(d.total_dofs()), d)
    u, st = geo.ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-12).solve(Kb, fb)
    exact = np.stack([exx * xyz[:, 0], exx * xyz[:, 1], ezz * xyz[:, 2]], axis=1).ravel()
    assert st.converged and np.abs(u - exact).max() <= 1e-6 * np.abs(exact).max()
    op = geo.ElasticityOperator(mesh, d, mat)
    for prec in ("fp64", "mixed"):
        um, sm = op.forward(np.zeros(d.total_dofs()),
                            geo.ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-12).with_precision(prec))
        assert sm.converged and np.abs(um - exact).max() <= 1e-6 * np.abs(exact).max()


def test_halfspace_gravity_confined_compression(geo):
    """elasticity_halfspace_gravity.rs: u_z(z) ~ -(rho g / M)(H z - z^2/2), ~5% (lateral effects)."""
    lx, ly, lz, E, nu, rho, g = 100e3, 100e3, 50e3, 100e9, 0.25, 3000.0, 9.81
    mesh = geo.ImprovedMeshGenerator.generate_cube(6, 6, 8, lx, ly, lz)
    xyz = mesh.nodes
    d = geo.DofManager(mesh.num_nodes(), 3)
    for i, (x, y, z) in enumerate(xyz):
        if abs(z) < 1.0:
            d.set_dirichlet(d.global_dof(i, 2), 0.0)
            if abs(x) < 1.0 and abs(y) < 1.0:
                d.set_dirichlet(d.global_dof(i, 0), 0.0)
                d.set_dirichlet(d.global_dof(i, 1), 0.0)
        if abs(x) < 1.0 or abs(x - lx) < 1.0:
            d.set_dirichlet(d.global_dof(i, 0), 0.0)
        if abs(y) < 1.0 or abs(y - ly) < 1.0:
            d.set_dirichlet(d.global_dof(i, 1), 0.0)
    op = geo.ElasticityOperator(mesh, d, geo.IsotropicElasticity(E, nu))
    f = geo.Assembler.assemble_gravity_load(mesh, d, rho, [0, 0, -g])
    u, st = op.forward(f, geo.ConjugateGradient().with_max_iterations(20000).with_tolerance(1e-10)
                       .with_precision("mixed"))
    assert st.converged
    M = E * (1 - nu) / ((1 + nu) * (1 - 2 * nu))
    top = np.abs(xyz[:, 2] - lz) < 1.0
    uz = u[2::3][top].mean()
    ana = -(rho * g / M) * (lz * lz - lz * lz / 2)
    assert abs(uz - ana) / abs(ana) < 0.1
